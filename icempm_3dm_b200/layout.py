"""Memory layouts and constants shared with the reference, without loading
the library: the SimParams3D parameter block (the reference's field order and
C types), the particle SoA row indices, the status bits, the precision modes
and the status codes of include/icempm_b200.h.

Importing this module (or icempm_3dm_b200.generator, which builds synthetic
inputs on it) loads no shared library; icempm_3dm_b200._lib binds the CUDA
library itself.
"""
import ctypes

# Row indices of the particle SoA (parameters_sim_3d.h:29-38).
IDX_UTILITY, IDX_P, IDX_Q, IDX_JP_INV = 0, 1, 2, 3
POSX, VELX, FE00, BP00 = 4, 7, 10, 19
N_PTS_ARRAYS = 28

STATUS_CRUSHED = 0x10000
STATUS_DISABLED = 0x20000
STATUS_LIQUID = 0x40000

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP64_SVD64 = 2

ACCUM_FLOAT = 0      # mixed P2G: FP32 float4 atomics (default)
ACCUM_FIXED = 1      # mixed P2G: 64-bit fixed point, order-independent sums

ERR_NAMES = {
    0: "ok", 5: "receive overflow",
    70: "particle outside grid (-x)", 71: "particle outside grid (-y)", 72: "particle outside grid (-z)",
    73: "particle outside grid (+x)", 74: "particle outside grid (+y)", 75: "particle outside grid (+z)",
    100: "CUDA runtime error", 101: "invalid argument", 102: "capacity exceeded", 103: "no suitable CUDA device",
    104: "configuration file not found", 105: "configuration file is not JSON / wrong key type",
    106: "config parameter missing (InputRawPoints)", 107: "cell key outside the grid",
    108: "call out of order", 109: "size beyond the fixed scratch of the allocation-free sort",
}


class SimParams3D(ctypes.Structure):
    """Same field order and C types as the reference's SimParams3D
    (simulation/parameters_sim_3d.h:40-90) and include/sim_params_3d.h."""
    _fields_ = [
        ("SetupType", ctypes.c_int),
        ("nPtsTotal", ctypes.c_int),
        ("GridXTotal", ctypes.c_int), ("GridY", ctypes.c_int), ("GridZ", ctypes.c_int),
        ("IndenterSubdivisions", ctypes.c_int),
        ("DomainDimensionX", ctypes.c_double),
        ("InitialTimeStep", ctypes.c_double), ("SimulationEndTime", ctypes.c_double),
        ("SimulationTime", ctypes.c_double),
        ("UpdateEveryNthStep", ctypes.c_int),
        ("SnapshotPeriod", ctypes.c_int),
        ("SimulationStep", ctypes.c_int),
        ("Gravity", ctypes.c_double), ("Density", ctypes.c_double), ("WaterDensity", ctypes.c_double),
        ("PoissonsRatio", ctypes.c_double), ("YoungsModulus", ctypes.c_double),
        ("DragGlobal", ctypes.c_double),
        ("lambda_", ctypes.c_double), ("mu", ctypes.c_double), ("kappa", ctypes.c_double),
        ("IceCompressiveStrength", ctypes.c_double), ("IceTensileStrength", ctypes.c_double),
        ("IceShearStrength", ctypes.c_double), ("IceTensileStrength2", ctypes.c_double),
        ("NACC_beta", ctypes.c_double),
        ("DP_tan_phi", ctypes.c_double), ("DP_threshold_p", ctypes.c_double),
        ("GrainVariability", ctypes.c_double),
        ("IndDiameter", ctypes.c_double), ("IndRSq", ctypes.c_double), ("IndVelocity", ctypes.c_double),
        ("IndDepth", ctypes.c_double),
        ("cellsize", ctypes.c_double),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double),
        ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("BlockCutout", ctypes.c_double * 3),
        ("ParticleVolume", ctypes.c_double), ("ParticleMass", ctypes.c_double),
        ("ParticleViewSize", ctypes.c_double), ("LiquidParticleMass", ctypes.c_double),
        ("indenter_x", ctypes.c_double), ("indenter_x_initial", ctypes.c_double),
        ("indenter_y", ctypes.c_double), ("indenter_y_initial", ctypes.c_double),
        ("Volume", ctypes.c_double),
        ("nPartitions", ctypes.c_int),
        ("GridHaloSize", ctypes.c_int),
        ("PointTransferFrequency", ctypes.c_int),
        ("VectorCapacity_transfer", ctypes.c_int),
        ("ExtraSpaceForIncomingPoints", ctypes.c_double),
        ("PointsTransferBufferFraction", ctypes.c_double),
        ("RebalanceThresholdFreeSpaceRemaining", ctypes.c_double),
        ("RebalanceThresholdDisabledPercentage", ctypes.c_double),
        ("dt_vol_Dpinv", ctypes.c_double), ("dt_Gravity", ctypes.c_double), ("vmax", ctypes.c_double),
        ("vmax_squared", ctypes.c_double),
        ("gbOffset", ctypes.c_int),
        ("cellsize_inv", ctypes.c_double), ("Dp_inv", ctypes.c_double),
        ("tpb_P2G", ctypes.c_int), ("tpb_Upd", ctypes.c_int), ("tpb_G2P", ctypes.c_int),
        ("animation_threshold_pos", ctypes.c_double),
    ]

    def copy(self):
        c = SimParams3D()
        ctypes.pointer(c)[0] = self
        return c
