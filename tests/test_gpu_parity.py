"""GPU parity of the FP64 step against the CPU oracle (restatement of
simulation/mpm_kernels.cuh), called through the C-ABI.

Tolerances: FP64 kernels differ from the oracle only by summation order of
the grid atomics and by fused multiply-adds, so single-step results agree
to ~1e-12 relative; the cell-key sort and the FP32 SVD are bit-exact.
"""
import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_FP64_SVD64, PRECISION_MIXED
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import (BP00, IDX_JP_INV, IDX_P, IDX_Q, IDX_UTILITY, LIB, POSX, STATUS_DISABLED, check,
                                  dptr)
from oracle import pyoracle as po
from tests.helpers import close, perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.gpu

STATE_ROWS = list(range(POSX, BP00 + 9)) + [IDX_JP_INV]


def gpu_svd(A, mode):
    count = A.shape[0]
    A = np.ascontiguousarray(A, dtype=np.float64)
    U = np.zeros((count, 9)); S = np.zeros((count, 3)); V = np.zeros((count, 9))
    check(LIB.mpm_testing_svd3x3(mode, dptr(A), count, dptr(U), dptr(S), dptr(V), 0), "svd")
    return U.reshape(-1, 3, 3), S, V.reshape(-1, 3, 3)


def test_svd_f32_bit_exact_vs_oracle_and_golden():
    rng = np.random.default_rng(3)
    A = np.concatenate([rng.standard_normal((2000, 9)),
                        (np.eye(3).reshape(9) + 1e-3 * rng.standard_normal((2000, 9))),
                        (np.eye(3).reshape(9) + 1e-6 * rng.standard_normal((1000, 9)))])
    U, S, V = gpu_svd(A, 0)
    for k in range(A.shape[0]):
        u, s, v = po.svd(A[k].reshape(3, 3))
        assert np.array_equal(u, U[k]) and np.array_equal(s, S[k]) and np.array_equal(v, V[k]), k
    g = np.load(po_golden_path())
    U2, S2, V2 = gpu_svd(g["A"], 0)
    bad = [k for k in range(g["A"].shape[0])
           if not (np.array_equal(U2[k].reshape(9), g["U"][k]) and np.array_equal(S2[k], g["S"][k])
                   and np.array_equal(V2[k].reshape(9), g["V"][k]))]
    assert not bad, (len(bad), bad[:10], [g["A"][k].tolist() for k in bad[:3]])


def po_golden_path():
    import os
    return os.path.join(os.path.dirname(__file__), "golden", "svd_ref.npz")


def test_svd_f64_accuracy():
    rng = np.random.default_rng(4)
    A = np.concatenate([rng.standard_normal((500, 9)), np.eye(3).reshape(9) + 1e-4 * rng.standard_normal((500, 9))])
    U, S, V = gpu_svd(A, 1)
    for k in range(A.shape[0]):
        R = U[k] @ np.diag(S[k]) @ V[k].T
        assert np.abs(R - A[k].reshape(3, 3)).max() < 1e-13 * max(1, np.abs(A[k]).max())
        assert np.abs(U[k].T @ U[k] - np.eye(3)).max() < 1e-13
        assert np.abs(V[k].T @ V[k] - np.eye(3)).max() < 1e-13
        assert S[k][0] >= S[k][1] >= abs(S[k][2]) - 1e-15


def test_sort_permutation_bit_exact():
    prms, soa = perturbed_block(n=5000, seed=21)
    n = soa.shape[1]
    rng = np.random.default_rng(5)
    order = rng.permutation(n)
    soa = np.ascontiguousarray(soa[:, order])
    bits = util_bits(soa).copy()
    dis = rng.random(n) < 0.05
    bits[dis] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    # many ties: snap some particles to identical positions
    soa[POSX:POSX + 3, 1:200:2] = soa[POSX:POSX + 3, 0:199:2]
    perm = po.sort_permutation(prms, soa, n)
    with MPMHandle(prms, n) as h:
        h.upload(soa)
        assert h.sort() == 0
        ids = h.ids()
        out = h.download()
    assert ids.shape == perm.shape
    assert np.array_equal(ids, perm)
    assert np.array_equal(out, soa[:, perm])


def one_phase_step(prms, soa, record=True, p0=None, precision=PRECISION_FP64):
    n = soa.shape[1]
    with MPMHandle(prms, n, precision) as h:
        h.upload(soa)
        if p0 is not None:
            h.upload(soa, cohesion=p0 * prms.DP_tan_phi)
        h.reset_indenter_force_accumulator()
        h.reset_grid()
        h.p2g()
        g_p2g = h.grid()
        h.update_nodes(prms.indenter_x + 0.02, prms.indenter_y)
        g_upd = h.grid()
        h.g2p(record)
        out = h.download()
        sensor, total = h.sensors()
    return g_p2g, g_upd, out, sensor


def test_single_step_phases_match_oracle():
    prms, soa = perturbed_block(n=4000, seed=31)
    n = soa.shape[1]
    g_p2g, g_upd, out, sensor = one_phase_step(prms, soa)

    ref_grid, err = po.p2g(prms, soa, n)
    assert err == 0
    ok, rel = close(g_p2g[0], ref_grid[0], 1e-12)
    assert ok, rel
    for c in range(1, 4):
        ok, rel = close(g_p2g[c], ref_grid[c], 1e-9, 1e-12)
        assert ok, (c, rel)

    f, ref_sensor = po.update_nodes(prms, ref_grid, prms.indenter_x + 0.02, prms.indenter_y)
    assert np.abs(f).max() > 0, "indenter should touch the block"
    for c in range(4):
        ok, rel = close(g_upd[c], ref_grid[c], 1e-9, 1e-12)
        assert ok, (c, rel)
    norm = prms.UpdateEveryNthStep * prms.cellsize ** 2
    ok, rel = close(sensor, ref_sensor / norm, 1e-9, 1e-12)
    assert ok, rel

    ref = soa.copy()
    assert po.g2p(prms, ref, n, ref_grid, record_pq=True) == 0
    assert np.array_equal(util_bits(out), util_bits(ref))
    for r in STATE_ROWS + [IDX_P, IDX_Q]:
        ok, rel = close(out[r], ref[r], 1e-9, 1e-12)
        assert ok, (r, rel)


def test_step_driver_matches_oracle_and_phases():
    prms, soa = perturbed_block(n=3000, seed=41, ind_velocity=0.5)
    n = soa.shape[1]
    steps = 40
    with MPMHandle(prms, n) as h:
        h.upload(soa)
        hist = h.step(steps)
        out = h.download()
        p_after = h.params()
    sim = po.OracleSim(prms, soa, n)
    ref_hist, err = sim.step(steps)
    assert err == 0
    assert p_after.SimulationStep == steps
    assert abs(p_after.SimulationTime - sim.prms.SimulationTime) < 1e-15
    assert np.abs(ref_hist).max() > 0
    ok, rel = close(hist, ref_hist, 1e-7, 1e-9)
    assert ok, rel
    assert np.array_equal(util_bits(out), util_bits(sim.soa))
    for r in STATE_ROWS:
        ok, rel = close(out[r], sim.soa[r], 1e-7, 1e-10)
        assert ok, (r, rel)


def test_per_particle_cohesion_matches_oracle():
    prms, soa = perturbed_block(n=3000, seed=51, crushed_frac=0.5)
    n = soa.shape[1]
    rng = np.random.default_rng(9)
    cohesion = 3e5 * np.exp(0.3 * rng.standard_normal(n))
    p0 = cohesion / prms.DP_tan_phi
    _, _, out, _ = one_phase_step(prms, soa, p0=p0)
    ref_grid, _ = po.p2g(prms, soa, n)
    po.update_nodes(prms, ref_grid, prms.indenter_x + 0.02, prms.indenter_y)
    ref = soa.copy()
    po.g2p(prms, ref, n, ref_grid, record_pq=True, p0=p0)
    assert np.array_equal(util_bits(out), util_bits(ref))
    for r in STATE_ROWS:
        ok, rel = close(out[r], ref[r], 1e-9, 1e-12)
        assert ok, (r, rel)


def test_fp64_svd_mode_matches_oracle_f64():
    prms, soa = perturbed_block(n=3000, seed=61, crushed_frac=0.6)
    n = soa.shape[1]
    _, _, out, _ = one_phase_step(prms, soa, precision=PRECISION_FP64_SVD64)
    ref_grid, _ = po.p2g(prms, soa, n)
    po.update_nodes(prms, ref_grid, prms.indenter_x + 0.02, prms.indenter_y)
    ref = soa.copy()
    po.g2p(prms, ref, n, ref_grid, record_pq=True, svd_mode=1)
    for r in STATE_ROWS:
        ok, rel = close(out[r], ref[r], 1e-9, 1e-12)
        assert ok, (r, rel)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
@pytest.mark.parametrize("axis,side,code", [(0, -1, 70), (1, -1, 71), (2, -1, 72), (0, 1, 73), (1, 1, 74),
                                             (2, 1, 75)])
def test_out_of_grid_error_codes(axis, side, code, precision):
    prms, soa, _ = gen.small_block(n=500, seed=3)
    dims = [prms.GridXTotal + 2 * prms.GridHaloSize, prms.GridY, prms.GridZ]
    h_ = prms.cellsize
    halo = prms.GridHaloSize * h_ if axis == 0 else 0.0
    soa[POSX + axis, 7] = (-0.8 * h_ if side < 0 else (dims[axis] - 1.2) * h_) - halo
    n = soa.shape[1]
    ref_grid, err = po.p2g(prms, soa, n)
    assert err == code
    with MPMHandle(prms, n, precision) as h:
        h.upload(soa)
        r = h.step(1, raise_on_error=False, want_forces=False)
        assert r == code
        assert h.error() == code
