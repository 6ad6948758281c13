"""The oracle pinned against the reference's own kernels.

oracle/_ref/libref_mpm.so is simulation/mpm_kernels.cuh of the reference,
compiled unmodified as host C++ (oracle/ref_kernels.cpp over the Eigen-API
stand-in of oracle/refshim/) and driven serially in index order by
oracle.pyoracle.RefSim. The oracle (oracle/mpm_oracle.cpp, the checker of
every GPU parity test) must agree with it phase by phase and over runs of
substeps, on inputs that reach every branch of the step: elastic, crushed in
compression and tension (Jp_inv < 1), strongly strained, liquid particles,
per-grain strength variability, indenter contact, the water-tank setup with
drag, and a grid with halo slabs.

Tolerances: one phase 1e-13 of each field's largest magnitude (the two differ
only in the order of rounded operations: Eigen's expression order against
the oracle's explicit 3x3 arithmetic), 1e-12 for the recorded trial P and Q
(J^2 - 1 near J = 1), 1e-11 for the indenter sensor bins (differences of
nearly equal velocities); 30 substeps 1e-11 (the same
rounding, carried through the run; C 1e-10, a difference quotient over h of
node velocities); integer status words bit for bit.

One reference behaviour is excluded from the comparison, on purpose: for
liquid particles partition_kernel_g2p computes no trial p, q (ComputePQ runs
in the solid branch only, mpm_kernels.cuh:316-327) but stores p.p_tr and
p.q_tr on record steps all the same (:347-351), i.e. whatever the
uninitialised fields hold. The oracle and the product write 0 there.
"""
import ctypes

import numpy as np
import pytest

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200.layout import IDX_UTILITY, POSX, STATUS_LIQUID, SimParams3D
from oracle import params as oracle_params
from oracle import pyoracle as po
from tests.helpers import perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.skipif(po.ref_mpm_lib() is None,
                                reason="oracle/_ref/libref_mpm.so not built (the reference tree is absent)")

FIELDS = (("Jp_inv", 3, 4), ("x", 4, 7), ("v", 7, 10), ("F", 10, 19), ("C", 19, 28))


def cases():
    """(name, prms, soa) inputs that reach every branch of the step. The
    parameter blocks come from the oracle's own restatement of the
    reference's SimParams3D routines. Cases with liquid particles use the
    water tank's stiffness (E = 1e8, as input_data/tank1b.json): at 5e8 and
    dt = 1e-5 the water model is unstable within tens of substeps, and any
    rounding difference then grows by a factor ~3 per substep."""
    ops = oracle_params.OPS
    out = []
    prms, soa = perturbed_block(n=2500, seed=11, ops=ops)
    out.append(("elastic+crushed+tension", prms, soa))
    prms, soa = perturbed_block(n=2500, seed=12, liquid_frac=0.2, youngs=1e8, ops=ops)
    out.append(("liquid", prms, soa))
    prms, soa = perturbed_block(n=2500, seed=13, crushed_frac=0.3, tension_frac=0.1, ops=ops)
    prms.GrainVariability = 0.5
    rng = np.random.default_rng(13)
    bits = util_bits(soa).copy()
    bits |= rng.integers(0, 1000, soa.shape[1])
    soa[IDX_UTILITY] = util_as_double(bits)
    out.append(("grain variability", prms, soa))
    prms, soa = perturbed_block(n=2000, seed=14, liquid_frac=0.5, youngs=1e8, ops=ops)
    prms.SetupType = 2
    prms.DragGlobal = 0.01
    out.append(("water tank + drag", prms, soa))
    prms, soa, _ = gen.small_block(n=2000, seed=15, halo=4, ops=ops)
    rng = np.random.default_rng(15)
    soa[7:10] = 0.1 * rng.standard_normal((3, soa.shape[1]))
    soa[10:19] += 1e-3 * rng.standard_normal((9, soa.shape[1]))
    prms.indenter_x_initial += 2 * prms.cellsize   # in contact from the first substep
    prms.indenter_x = prms.indenter_x_initial
    out.append(("halo slabs + contact", prms, soa))
    return out


CASES = cases()


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_parameter_block_layout_is_the_references():
    lib = po.ref_mpm_lib()
    assert lib.ref_sizeof_params() == ctypes.sizeof(SimParams3D)
    off = (ctypes.c_size_t * 12)()
    lib.ref_params_layout(off)
    names = ["SetupType", "GridXTotal", "InitialTimeStep", "mu", "IndRSq", "cellsize", "ParticleMass",
             "GridHaloSize", "dt_vol_Dpinv", "gbOffset", "tpb_G2P", "animation_threshold_pos"]
    assert list(off) == [getattr(SimParams3D, nm).offset for nm in names]


@pytest.mark.parametrize("name,prms,soa", CASES, ids=[c[0] for c in CASES])
def test_one_substep_phase_by_phase(name, prms, soa):
    n = soa.shape[1]
    ref = po.RefSim(prms, soa, n)
    ref._upload_params()
    ref.p2g()
    grid, err = po.p2g(prms, soa, n)
    assert err == 0 and ref.lib.ref_error() == 0
    assert rel(ref.grid[0], grid[0]) < 1e-13
    assert rel(ref.grid[1:], grid[1:]) < 1e-13

    f_ref = ref.update_nodes(prms.indenter_x, prms.indenter_y)
    f_or, sensor = po.update_nodes(prms, grid, prms.indenter_x, prms.indenter_y)
    assert rel(ref.grid[1:], grid[1:]) < 1e-13
    # a contact force is (v_old - v) m / dt of nearly equal velocities: the
    # cancellation scales the rounding up, hence 1e-11 for the sensor bins
    assert rel(ref.step_sensor, sensor) < 1e-11 if np.any(sensor) else not np.any(ref.step_sensor)
    assert np.allclose(f_ref, f_or, rtol=1e-11, atol=1e-11 * max(np.abs(f_or).max(), 1e-300))

    out = np.array(soa)
    assert po.g2p(prms, out, n, grid, record_pq=True) == 0
    ref.g2p(True)
    assert np.array_equal(util_bits(ref.soa), util_bits(out))
    for fname, a, b in FIELDS:
        assert rel(ref.soa[a:b], out[a:b]) < 1e-13, fname
    # trial p = -kappa/2 (J^2 - 1) cancels near J = 1: 1e-12 for P and Q
    solid = (util_bits(out) & STATUS_LIQUID) == 0
    assert rel(ref.soa[1:3, solid], out[1:3, solid]) < 1e-12


@pytest.mark.parametrize("name,prms,soa", CASES, ids=[c[0] for c in CASES])
def test_thirty_substeps(name, prms, soa):
    n = soa.shape[1]
    ref = po.RefSim(prms, soa, n)
    orc = po.OracleSim(prms, soa, n)
    h_ref, e_ref = ref.step(30)
    h_or, e_or = orc.step(30)
    assert e_ref == 0 and e_or == 0
    assert rel(h_ref, h_or) < 1e-11
    assert np.array_equal(util_bits(ref.soa), util_bits(orc.soa))
    for fname, a, b in FIELDS:
        # C = 4/h sum w v (x_i - x_p): node-velocity rounding scaled by 1/h
        assert rel(ref.soa[a:b], orc.soa[a:b]) < (1e-10 if fname == "C" else 1e-11), fname
    assert ref.prms.SimulationStep == orc.prms.SimulationStep == 30
    assert ref.prms.indenter_x == orc.prms.indenter_x


def test_crushing_branches_are_reached():
    """The cases above cross the failure surface in both branches and
    return-map in both branches of Wolper_Drucker_Prager."""
    prms, soa = CASES[0][1], CASES[0][2]
    n = soa.shape[1]
    before = (util_bits(soa) & 0x10000) != 0
    ref = po.RefSim(prms, soa, n)
    ref.step(1)
    after = (util_bits(ref.soa) & 0x10000) != 0
    assert (after & ~before).sum() > 0                    # newly crushed this substep
    assert (soa[3] < 1).sum() > 0                          # Jp_inv < 1: the tension branch
    assert np.abs(ref.soa[POSX:POSX + 3] - soa[POSX:POSX + 3]).max() > 0
