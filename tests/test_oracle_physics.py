"""Known-answer tests of the CPU oracle (restatement of mpm_kernels.cuh):
conservation, APIC exactness on affine velocity fields, the cell-key sort,
the Drucker-Prager return map landing on its yield surface, error codes, and
serial/OpenMP agreement. These pin the oracle where the reference ships no
golden outputs."""
import numpy as np
import pytest

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import (BP00, FE00, IDX_P, IDX_Q, IDX_UTILITY, LIB, POSX, STATUS_CRUSHED, STATUS_DISABLED,
                                  VELX)
from oracle import pyoracle as po
from tests.helpers import perturbed_block, util_as_double, util_bits


def quiet(prms):
    """No gravity, indenter far away."""
    p = prms.copy()
    p.Gravity = 0.0
    LIB.mpm_params_compute_helper_variables(p)
    p.indenter_x = -10.0
    p.indenter_y = -10.0
    return p


def interior_block(n=2000, seed=3):
    prms, soa, _ = gen.small_block(n=n, seed=seed)
    return quiet(prms), soa


def test_p2g_conserves_mass_and_momentum():
    prms, soa = perturbed_block(n=3000, seed=5)
    n = soa.shape[1]
    grid, err = po.p2g(prms, soa, n)
    assert err == 0
    assert grid[0].sum() == pytest.approx(n * prms.ParticleMass, rel=1e-13)
    mom = prms.ParticleMass * soa[VELX:VELX + 3].sum(axis=1)
    for c in range(3):
        assert grid[1 + c].sum() == pytest.approx(mom[c], abs=1e-12 * np.abs(grid[1 + c]).sum())


def test_single_particle_at_rest():
    prms, soa = interior_block(n=500)
    one = np.ascontiguousarray(soa[:, 250:251])
    grid, err = po.p2g(prms, one, 1)
    assert err == 0
    assert grid[0].sum() == pytest.approx(prms.ParticleMass, rel=1e-14)
    assert (grid[0] > 0).sum() == 27
    assert np.abs(grid[1:]).max() < 1e-20


@pytest.mark.parametrize("affine", [False, True])
def test_apic_reproduces_affine_velocity(affine):
    prms, soa = interior_block(n=4000)
    n = soa.shape[1]
    rng = np.random.default_rng(1)
    v0 = np.array([0.01, -0.02, 0.015])
    A = 0.05 * rng.standard_normal((3, 3)) if affine else np.zeros((3, 3))
    x = soa[POSX:POSX + 3]
    soa[VELX:VELX + 3] = v0[:, None] + A @ x
    soa[BP00:BP00 + 9] = A.reshape(9, 1)
    grid, err = po.p2g(prms, soa, n)
    po.update_nodes(prms, grid, prms.indenter_x, prms.indenter_y)
    # particles whose stencil sees no wall node keep the affine field exactly
    h = prms.cellsize
    base = np.floor(x / h - 0.5).astype(int)
    lo = np.array([3, 3, 3])
    hi = np.array([prms.GridXTotal - 4, prms.GridY - 4, prms.GridZ - 4])
    free = np.all((base >= lo[:, None]) & (base + 2 <= hi[:, None]), axis=0)
    assert free.sum() > 100
    out = soa.copy()
    assert po.g2p(prms, out, n, grid) == 0
    dt = prms.InitialTimeStep
    vref = v0[:, None] + A @ x
    assert np.abs(out[VELX:VELX + 3][:, free] - vref[:, free]).max() < 1e-14
    assert np.abs(out[BP00:BP00 + 9][:, free] - A.reshape(9, 1)).max() < 1e-11
    assert np.abs(out[POSX:POSX + 3][:, free] - (x + vref * dt)[:, free]).max() < 1e-15
    F = (np.eye(3) + dt * A).reshape(9)
    assert np.abs(out[FE00:FE00 + 9][:, free] - F[:, None]).max() < 1e-14


def test_sort_is_stable_by_reference_cell_key():
    prms, soa = perturbed_block(n=5000, seed=8)
    n = soa.shape[1]
    rng = np.random.default_rng(0)
    soa = np.ascontiguousarray(soa[:, rng.permutation(n)])
    bits = util_bits(soa).copy()
    dis = rng.random(n) < 0.1
    bits[dis] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    perm = po.sort_permutation(prms, soa, n)
    assert len(perm) == n - dis.sum()
    assert not dis[perm].any()
    x = soa[POSX:POSX + 3, perm] * prms.cellsize_inv + 0.5
    keys = (x[0].astype(int) * prms.GridY * prms.GridZ + x[1].astype(int) * prms.GridZ + x[2].astype(int))
    for k in range(len(perm)):
        assert keys[k] == po.cell_key(prms, *soa[POSX:POSX + 3, perm[k]])
    assert np.all(np.diff(keys) >= 0)
    ties = np.diff(keys) == 0
    assert np.all(np.diff(perm.astype(np.int64))[ties] > 0)     # stable


def trial_pq(prms, F):
    J = np.linalg.det(F)
    b = F @ F.T
    d = b - np.trace(b) / 3 * np.eye(3)
    p = -0.5 * prms.kappa * (J * J - 1)
    q = np.sqrt(1.5) * prms.mu * (J * J) ** (-1 / 3) * np.linalg.norm(d)
    return p, q


@pytest.mark.parametrize("svd_mode", [0, 1])
def test_return_map_lands_on_yield_surface(svd_mode):
    prms, soa = interior_block(n=3000)
    n = soa.shape[1]
    rng = np.random.default_rng(7)
    E = 0.02 * rng.standard_normal((9, n))
    # compressive, deviatoric trial states of crushed points
    soa[FE00:FE00 + 9] = np.eye(3).reshape(9, 1) + E - 0.004 * np.eye(3).reshape(9, 1)
    soa[IDX_UTILITY] = util_as_double(np.full(n, STATUS_CRUSHED))
    grid = np.zeros((4, po.grid_nodes(prms)))
    out = soa.copy()
    po.g2p(prms, out, n, grid, record_pq=True, svd_mode=svd_mode)   # zero grid: F unchanged before the map
    p0 = prms.DP_threshold_p
    checked = 0
    tol = 2e-5 if svd_mode == 0 else 1e-9
    for k in range(0, n, 7):
        F_tr = soa[FE00:FE00 + 9, k].reshape(3, 3)
        p_tr, q_tr = trial_pq(prms, F_tr)
        F_new = out[FE00:FE00 + 9, k].reshape(3, 3)
        p_new, q_new = trial_pq(prms, F_new)
        if p_tr < -p0:
            s = np.linalg.svd(F_new, compute_uv=False)
            assert np.allclose(s, s[0], rtol=1e-6)
            continue
        pmax, pmin, qmax = prms.IceCompressiveStrength, -prms.IceTensileStrength, prms.IceShearStrength
        q_lim = 0 if p_tr > pmax else min(2 * np.sqrt((pmax - p_tr) * (p_tr - pmin)) * qmax / (pmax - pmin),
                                          (p_tr + p0) * prms.DP_tan_phi)
        if q_tr >= q_lim:
            # the projection keeps the mean of Sigma^2 and scales its
            # deviator to q_n_1 measured with the trial J (mpm_kernels.cuh:532-542)
            s_tr = np.linalg.svd(F_tr, compute_uv=False) ** 2
            s_new = np.linalg.svd(F_new, compute_uv=False) ** 2
            assert s_new.mean() == pytest.approx(s_tr.mean(), rel=tol)
            J_tr = np.linalg.det(F_tr)
            q_dev = np.sqrt(1.5) * prms.mu * (J_tr * J_tr) ** (-1 / 3) * np.linalg.norm(s_new - s_new.mean())
            assert q_dev == pytest.approx(q_lim, rel=50 * tol, abs=tol * prms.mu * 1e-3)
            checked += 1
        else:
            assert np.abs(F_new - F_tr).max() == 0
    assert checked > 50


def test_failure_surface_sets_crushed_bit_and_records_pq():
    prms, soa = interior_block(n=2000)
    n = soa.shape[1]
    soa[FE00:FE00 + 9] = np.eye(3).reshape(9, 1)
    soa[FE00 + 1, :n // 2] = 0.2      # strong shear on half of the points
    grid = np.zeros((4, po.grid_nodes(prms)))
    out = soa.copy()
    po.g2p(prms, out, n, grid, record_pq=True)
    crushed = (util_bits(out) & STATUS_CRUSHED) != 0
    assert crushed[:n // 2].all() and not crushed[n // 2:].any()
    p, q = trial_pq(prms, soa[FE00:FE00 + 9, 0].reshape(3, 3))
    assert out[IDX_P, 0] == pytest.approx(p, rel=1e-12) and out[IDX_Q, 0] == pytest.approx(q, rel=1e-12)


@pytest.mark.parametrize("axis,side,code", [(0, -1, 70), (1, -1, 71), (2, -1, 72), (0, 1, 73), (1, 1, 74),
                                             (2, 1, 75)])
def test_error_codes(axis, side, code):
    prms, soa, _ = gen.small_block(n=400, seed=3)
    dims = [prms.GridXTotal + 2 * prms.GridHaloSize, prms.GridY, prms.GridZ]
    h = prms.cellsize
    halo = prms.GridHaloSize * h if axis == 0 else 0.0
    soa[POSX + axis, 5] = (-0.8 * h if side < 0 else (dims[axis] - 1.2) * h) - halo
    _, err = po.p2g(prms, soa, soa.shape[1])
    assert err == code


def test_openmp_matches_serial():
    prms, soa = perturbed_block(n=4000, seed=9)
    n = soa.shape[1]
    a = po.OracleSim(prms, soa, n, nthreads=1)
    b = po.OracleSim(prms, soa, n, nthreads=4)
    ha, _ = a.step(5)
    hb, _ = b.step(5)
    assert np.allclose(ha, hb, rtol=1e-9, atol=1e-9 * np.abs(ha).max())
    assert np.abs(a.soa[POSX:POSX + 3] - b.soa[POSX:POSX + 3]).max() < 1e-13
