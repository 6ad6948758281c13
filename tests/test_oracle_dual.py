"""The oracle's FP64 dual-number forward mode (or_dual_steps, or_svd3x3_dual)
against central finite differences of the oracle itself, on the CPU.

The dual forward mode is the second, independent check of the product's
hand-written adjoint (tests/test_gpu_adjoint.py); this file pins it first.
Its value part must equal the oracle bit for bit (same arithmetic, the
scalar type only carries a tangent); its tangents must match central
differences to 1e-5 relative (truncation and rounding of the differences).
"""
import numpy as np
import pytest

from icempm_3dm_b200._lib import BP00, FE00, IDX_JP_INV, LIB, POSX, VELX
from oracle import pyoracle as po
from tests.helpers import perturbed_block


def test_svd_dual_matches_finite_differences():
    rng = np.random.default_rng(12)
    for k in range(200):
        A = np.eye(3) + (0.3 if k % 2 else 1e-3) * rng.standard_normal((3, 3))
        dA = rng.standard_normal((3, 3))
        (U, S, V), (dU, dS, dV) = po.svd_dual(A, dA)
        U0, S0, V0 = po.svd(A, "f64")
        assert np.array_equal(U, U0) and np.array_equal(S, S0) and np.array_equal(V, V0)
        # near-degenerate singular values (gap ~1e-3) make dU, dV large and
        # the central difference's truncation error grows with h / gap
        h = 1e-6 if k % 2 else 1e-9
        Up, Sp, Vp = po.svd(A + h * dA, "f64")
        Um, Sm, Vm = po.svd(A - h * dA, "f64")
        for d, p, m in ((dS, Sp, Sm), (dU, Up, Um), (dV, Vp, Vm)):
            fd = (p - m) / (2 * h)
            assert np.abs(d - fd).max() < 1e-5 * max(1.0, np.abs(fd).max()), k


def small_case(n=600, seed=17):
    prms, soa = perturbed_block(n=n, seed=seed, crushed_frac=0.4, strong_frac=0.15, ind_velocity=0.5,
                                dims=(0.10, 0.06, 0.06))
    rng = np.random.default_rng(seed)
    p0 = 3e5 * np.exp(0.3 * rng.standard_normal(soa.shape[1])) / prms.DP_tan_phi
    return prms, soa, p0


def oracle_loss(prms, soa, p0, wgt, nsteps):
    sim = po.OracleSim(prms, soa, soa.shape[1], p0=p0, svd_mode=1)
    hist, err = sim.step(nsteps)
    assert err == 0
    return float(np.sum(wgt * hist))


def with_E(prms, E):
    p = prms.copy()
    p.YoungsModulus = E
    LIB.mpm_params_compute_camclay(p)
    LIB.mpm_params_compute_helper_variables(p)
    return p


@pytest.mark.parametrize("direction", ["E", "cohesion", "velocity", "position", "F", "C"])
def test_dual_steps_match_finite_differences(direction):
    nsteps = 6
    prms, soa, p0 = small_case()
    n = soa.shape[1]
    rng = np.random.default_rng(5)
    wgt = rng.standard_normal((nsteps, 3))
    wgt[:, 2] = 0.0
    dsoa = np.zeros_like(soa)
    dp0 = None
    dE = 0.0
    if direction == "E":
        dE = 1.0
    elif direction == "cohesion":
        dp0 = p0 * rng.standard_normal(n)
    else:
        row, rows, scale = {"velocity": (VELX, 3, 0.05), "position": (POSX, 3, 1e-3),
                            "F": (FE00, 9, 1e-3), "C": (BP00, 9, 5.0)}[direction]
        dsoa[row:row + rows] = scale * rng.standard_normal((rows, n))

    hist, dhist, _, _ = po.dual_steps(prms, soa, nsteps, dsoa=dsoa, p0=p0, dp0=dp0, dE=dE)
    assert np.array_equal(hist, po.OracleSim(prms, soa, n, p0=p0, svd_mode=1).step(nsteps)[0])
    tangent = float(np.sum(wgt * dhist))

    # the force sums cancel strongly: small steps are rounding-bound, the
    # state directions converge to the tangent at eps ~ 1e-4 of their scale
    eps = 1e-6 if direction in ("E", "cohesion") else 1e-4
    if direction == "E":
        E = prms.YoungsModulus
        fd = (oracle_loss(with_E(prms, E * (1 + eps)), soa, p0, wgt, nsteps) -
              oracle_loss(with_E(prms, E * (1 - eps)), soa, p0, wgt, nsteps)) / (2 * eps * E)
    elif direction == "cohesion":
        fd = (oracle_loss(prms, soa, p0 + eps * dp0, wgt, nsteps) -
              oracle_loss(prms, soa, p0 - eps * dp0, wgt, nsteps)) / (2 * eps)
    else:
        fd = (oracle_loss(prms, soa + eps * dsoa, p0, wgt, nsteps) -
              oracle_loss(prms, soa - eps * dsoa, p0, wgt, nsteps)) / (2 * eps)
    assert tangent != 0.0
    assert abs(tangent - fd) <= 1e-5 * abs(fd), (direction, tangent, fd)


def test_dual_jp_tangent_through_tension_branch():
    """Jp_inv enters only through the tension-cutoff test and its update in the
    return map; its tangent must flow through the final state. The direction
    moves only particles already in tension (Jp_inv < 1): at Jp_inv = 1 the
    test `Jp_inv < 1` switches and the state is not differentiable."""
    prms, soa, p0 = small_case(seed=23)
    dsoa = np.zeros_like(soa)
    tension = soa[IDX_JP_INV] < 0.999
    assert tension.sum() > 5
    dsoa[IDX_JP_INV, tension] = 1.0
    _, _, s, ds = po.dual_steps(prms, soa, 3, dsoa=dsoa, p0=p0)
    eps = 1e-7
    sim_p = po.OracleSim(prms, soa + eps * dsoa, soa.shape[1], p0=p0, svd_mode=1)
    sim_m = po.OracleSim(prms, soa - eps * dsoa, soa.shape[1], p0=p0, svd_mode=1)
    sim_p.step(3)
    sim_m.step(3)
    fd = (sim_p.soa[IDX_JP_INV] - sim_m.soa[IDX_JP_INV]) / (2 * eps)
    assert np.abs(ds[IDX_JP_INV]).max() > 0
    assert np.abs(ds[IDX_JP_INV] - fd).max() < 1e-6 * np.abs(fd).max()
