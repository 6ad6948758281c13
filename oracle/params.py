"""CPU ORACLE — test infrastructure, not product code.

The parameter routines of the reference's SimParams3D restated in Python, so
that the checker and the reference arm of bench.py can build a parameter
block without loading the product library:

  reset                      SimParams3D::Reset (parameters_sim_3d.cpp:5-62)
  compute_helper_variables   SimParams3D::ComputeHelperVariables (:65-86)
  compute_lame               SimParams3D::ComputeLame (:164-169)
  compute_camclay            SimParams3D::ComputeCamClayParams (:171-175)
  set_phi                    SimParams3D::SetPhi (parameters_sim_3d.h:100)

Each works on a ctypes SimParams3D (icempm_3dm_b200.layout, the reference's
field layout) in place, with the reference's double arithmetic in the same
order; int fields truncate as the reference's implicit conversions do.
tests/test_oracle_params.py checks them field by field against the
library's own routines.
"""
import math
from collections import namedtuple

PI = 3.14159265358979323846     # SimParams3D::pi (parameters_sim_3d.h:24)


def _to_int(x):
    """C conversion of a double to int (truncation toward zero)."""
    return int(math.trunc(x))


def set_phi(p, phi_degrees):
    p.DP_tan_phi = math.tan(phi_degrees * PI / 180.0)


def compute_lame(p):
    p.lambda_ = p.YoungsModulus * p.PoissonsRatio / ((1 + p.PoissonsRatio) * (1 - 2 * p.PoissonsRatio))
    p.mu = p.YoungsModulus / (2 * (1 + p.PoissonsRatio))
    p.kappa = p.mu * 2.0 / 3.0 + p.lambda_


def compute_camclay(p):
    compute_lame(p)
    p.NACC_beta = p.IceTensileStrength / p.IceCompressiveStrength


def compute_helper_variables(p):
    p.ParticleMass = p.ParticleVolume * p.Density
    p.LiquidParticleMass = p.ParticleVolume * p.WaterDensity
    # (int)(1.f/(200*InitialTimeStep)): the float 1 is promoted to double
    p.UpdateEveryNthStep = _to_int(1.0 / (200 * p.InitialTimeStep))
    p.cellsize = p.DomainDimensionX / p.GridXTotal
    p.cellsize_inv = 1.0 / p.cellsize
    p.Dp_inv = 4.0 / (p.cellsize * p.cellsize)
    p.IndRSq = p.IndDiameter * p.IndDiameter / 4.0
    p.dt_vol_Dpinv = p.InitialTimeStep * p.ParticleVolume * p.Dp_inv
    p.dt_Gravity = p.InitialTimeStep * p.Gravity
    p.vmax = 0.5 * p.cellsize / p.InitialTimeStep
    p.vmax_squared = p.vmax * p.vmax
    # nPtsTotal/nPartitions is an int division (truncating), then times a double
    q = abs(p.nPtsTotal) // abs(p.nPartitions)
    q = q if (p.nPtsTotal >= 0) == (p.nPartitions > 0) else -q
    p.VectorCapacity_transfer = _to_int(q * p.PointsTransferBufferFraction)
    p.gbOffset = p.GridZ * p.GridY * p.GridHaloSize
    p.IndenterSubdivisions = _to_int(PI * p.IndDiameter / p.cellsize)


def reset(p):
    p.nPtsTotal = 0
    p.SimulationEndTime = 12
    p.SimulationStep = 0
    p.SimulationTime = 0
    p.InitialTimeStep = 3.e-5
    p.YoungsModulus = 5.e8
    p.GridXTotal = 128
    p.GridY = 55
    p.GridZ = 55
    p.ParticleViewSize = 2.5     # 2.5f is exact in float
    p.DomainDimensionX = 3.33
    p.PoissonsRatio = 0.3
    p.Gravity = 9.81
    p.Density = 916
    p.WaterDensity = 1000
    p.DragGlobal = 0
    p.IndDiameter = 0.324
    p.IndVelocity = 0.2
    p.IndDepth = 0.25
    p.IceCompressiveStrength = 100e6
    p.IceTensileStrength = 10e6
    p.IceShearStrength = 6e6
    p.IceTensileStrength2 = 5e6
    set_phi(p, 45)
    p.DP_threshold_p = 1e2
    p.tpb_P2G = 256
    p.tpb_Upd = 512
    p.tpb_G2P = 128
    p.indenter_x = p.indenter_x_initial = p.indenter_y = p.indenter_y_initial = 0
    p.SetupType = 0
    p.GrainVariability = 0.50
    p.GridHaloSize = 15
    p.ExtraSpaceForIncomingPoints = 0.2
    p.PointsTransferBufferFraction = 0.05
    p.nPartitions = 4
    p.RebalanceThresholdFreeSpaceRemaining = 0.10
    p.RebalanceThresholdDisabledPercentage = 0.05
    p.PointTransferFrequency = 2
    p.SnapshotPeriod = 100
    p.animation_threshold_pos = 1e-3
    compute_lame(p)
    compute_camclay(p)
    compute_helper_variables(p)


ParamOps = namedtuple("ParamOps", "reset set_phi compute_camclay compute_helper_variables")

# the routine set icempm_3dm_b200.generator takes as `ops`
OPS = ParamOps(reset, set_phi, compute_camclay, compute_helper_variables)
