"""Adjoint of the FP64 step (mpm_adjoint_forward / mpm_adjoint_backward)
for the gradient of a linear functional of the indenter force history with
respect to per-particle cohesion, Young's modulus and the initial particle
state, checked two ways:
  - against central finite differences through the GPU forward step, to
    1e-3 relative (the required bound) on the largest gradient entries;
  - against the oracle's FP64 dual-number forward mode (or_dual_steps, pinned
    against finite differences in test_oracle_dual.py) along E, a random
    cohesion direction and a random direction in the initial state, to 1e-6
    relative (both are exact derivatives; they differ by FP64 rounding and the
    summation order of the grid atomics).
FP64 forward, FP64 SVD (the precision the adjoint differentiates).
"""
import ctypes

import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64_SVD64
from icempm_3dm_b200._lib import BP00, FE00, IDX_JP_INV, LIB, POSX, VELX, check, dptr
from oracle import pyoracle as po
from tests.helpers import perturbed_block

pytestmark = pytest.mark.gpu


def case(n=1500, seed=7):
    prms, soa = perturbed_block(n=n, seed=seed, crushed_frac=0.4, strong_frac=0.15, ind_velocity=0.5,
                                dims=(0.12, 0.08, 0.08))
    rng = np.random.default_rng(seed)
    cohesion = 3e5 * np.exp(0.3 * rng.standard_normal(soa.shape[1]))
    return prms, soa, cohesion


def loss(prms, soa, cohesion, wgt, nsteps):
    with MPMHandle(prms, soa.shape[1], PRECISION_FP64_SVD64) as h:
        h.upload(soa, cohesion=cohesion)
        hist = h.step(nsteps)
    return float(np.sum(wgt * hist))


def adjoint(prms, soa, cohesion, wgt, nsteps, every):
    n = soa.shape[1]
    with MPMHandle(prms, n, PRECISION_FP64_SVD64) as h:
        h.upload(soa, cohesion=cohesion)
        hist = np.zeros((nsteps, 3))
        check(LIB.mpm_adjoint_forward(h._h, nsteps, every, dptr(hist)), "adjoint forward")
        dc = np.zeros(n)
        dE = ctypes.c_double(0)
        w = np.ascontiguousarray(wgt, dtype=np.float64)
        check(LIB.mpm_adjoint_backward(h._h, dptr(w), dptr(dc), ctypes.byref(dE)), "adjoint backward")
        adj = np.zeros((25, n))
        check(LIB.mpm_adjoint_state(h._h, dptr(adj), n), "adjoint state")
    return float(np.sum(wgt * hist)), dc, dE.value, adj


def with_E(prms, E):
    p = prms.copy()
    p.YoungsModulus = E
    LIB.mpm_params_compute_camclay(p)
    LIB.mpm_params_compute_helper_variables(p)
    return p


@pytest.mark.parametrize("nsteps,every", [(1, 1), (8, 3)])
def test_adjoint_matches_finite_differences(nsteps, every):
    prms, soa, coh = case()
    rng = np.random.default_rng(1)
    wgt = rng.standard_normal((nsteps, 3))
    wgt[:, 2] = 0.0
    L0, dc, dE, adj = adjoint(prms, soa, coh, wgt, nsteps, every)
    assert L0 != 0.0
    assert L0 == pytest.approx(loss(prms, soa, coh, wgt, nsteps), rel=1e-9)
    print(f"\nL = {L0:.6e}, nonzero dL/dc: {np.count_nonzero(dc)} of {dc.size}")
    if nsteps == 1:
        # the force of a substep is measured in the grid update, before the
        # return map reads the cohesion: one substep does not depend on it
        assert not np.any(dc)
    else:
        assert np.count_nonzero(dc) > dc.size // 2
    report = []

    # Young's modulus
    eps = 1e-6
    E = prms.YoungsModulus
    fd = (loss(with_E(prms, E * (1 + eps)), soa, coh, wgt, nsteps) -
          loss(with_E(prms, E * (1 - eps)), soa, coh, wgt, nsteps)) / (2 * eps * E)
    report.append(("E", fd, dE))

    # cohesion of the particles with the largest gradients
    for i in np.argsort(-np.abs(dc))[:4]:
        if abs(dc[i]) == 0:
            continue
        cp, cm = coh.copy(), coh.copy()
        cp[i] *= 1 + 1e-4
        cm[i] *= 1 - 1e-4
        fd = (loss(prms, soa, cp, wgt, nsteps) - loss(prms, soa, cm, wgt, nsteps)) / (2e-4 * coh[i])
        report.append((f"c[{i}]", fd, dc[i]))

    # initial velocity and position of the particles with the largest velocity adjoints
    for row, off, h in ((VELX, 3, 1e-5), (POSX, 0, 1e-7)):
        g = adj[off:off + 3]
        i = int(np.argmax(np.abs(g).max(axis=0)))
        d = int(np.argmax(np.abs(g[:, i])))
        sp, sm = soa.copy(), soa.copy()
        sp[row + d, i] += h
        sm[row + d, i] -= h
        fd = (loss(prms, sp, coh, wgt, nsteps) - loss(prms, sm, coh, wgt, nsteps)) / (2 * h)
        report.append((f"row{row + d}[{i}]", fd, g[d, i]))

    print("\n".join(f"{name:>14s}  fd {fd: .9e}  adjoint {ad: .9e}" for name, fd, ad in report))
    assert all(abs(ad) > 0 for _, _, ad in report), report          # non-trivial gradients
    assert len(report) == (3 if nsteps == 1 else 7)
    bad = [(name, fd, ad) for name, fd, ad in report if abs(fd - ad) > 1e-3 * max(abs(fd), abs(ad), 1e-30)]
    assert not bad, report


# rows of mpm_adjoint_state -> rows of the particle SoA
ADJ_TO_SOA = ((0, POSX, 3), (3, VELX, 3), (6, BP00, 9), (15, FE00, 9), (24, IDX_JP_INV, 1))


def test_adjoint_matches_dual_number_forward_mode():
    nsteps, every = 8, 3
    prms, soa, coh = case()
    n = soa.shape[1]
    rng = np.random.default_rng(2)
    wgt = rng.standard_normal((nsteps, 3))
    wgt[:, 2] = 0.0
    L0, dc, dE, adj = adjoint(prms, soa, coh, wgt, nsteps, every)
    p0 = coh / prms.DP_tan_phi
    report = []

    hist, dhist, _, _ = po.dual_steps(prms, soa, nsteps, p0=p0, dE=1.0)
    assert float(np.sum(wgt * hist)) == pytest.approx(L0, rel=1e-7)
    report.append(("E", float(np.sum(wgt * dhist)), dE))

    r = coh * rng.standard_normal(n)
    _, dhist, _, _ = po.dual_steps(prms, soa, nsteps, p0=p0, dp0=r / prms.DP_tan_phi)
    report.append(("cohesion", float(np.sum(wgt * dhist)), float(r @ dc)))

    dsoa = np.zeros_like(soa)
    scale = {POSX: 1e-3, VELX: 0.05, BP00: 5.0, FE00: 1e-3}
    for row, rows in ((POSX, 3), (VELX, 3), (BP00, 9), (FE00, 9)):
        dsoa[row:row + rows] = scale[row] * rng.standard_normal((rows, n))
    tension = soa[IDX_JP_INV] < 0.999          # Jp_inv = 1 sits on the tension test's switch
    dsoa[IDX_JP_INV, tension] = 1e-3 * rng.standard_normal(int(tension.sum()))
    _, dhist, _, _ = po.dual_steps(prms, soa, nsteps, dsoa=dsoa, p0=p0)
    vjp = sum(float(np.sum(adj[a:a + k] * dsoa[s:s + k])) for a, s, k in ADJ_TO_SOA)
    report.append(("state", float(np.sum(wgt * dhist)), vjp))

    print("\n" + "\n".join(f"{name:>9s}  dual {t: .12e}  adjoint {a: .12e}" for name, t, a in report))
    for name, t, a in report:
        assert t != 0.0, name
        assert abs(t - a) <= 1e-6 * abs(t), (name, t, a)


def test_single_call_adjoint_equals_forward_then_backward():
    nsteps, every = 6, 2
    prms, soa, coh = case()
    n = soa.shape[1]
    wgt = np.random.default_rng(5).standard_normal((nsteps, 3))
    _, dc2, dE2, _ = adjoint(prms, soa, coh, wgt, nsteps, every)
    with MPMHandle(prms, n, PRECISION_FP64_SVD64) as h:
        h.upload(soa, cohesion=coh)
        dc = np.zeros(n)
        dE = ctypes.c_double(0)
        w = np.ascontiguousarray(wgt)
        check(LIB.mpm_adjoint(h._h, nsteps, every, dptr(w), dptr(dc), ctypes.byref(dE)), "mpm_adjoint")
    # two GPU runs differ only by the summation order of FP64 atomics
    assert np.allclose(dc, dc2, rtol=1e-8, atol=1e-8 * np.abs(dc2).max())
    assert dE.value == pytest.approx(dE2, rel=1e-8)


def test_mixed_forward_adjoint_follows_the_fp64_adjoint():
    """The calibration row's mixed forward: mpm_adjoint_forward on a mixed
    handle runs the mixed step (checkpoints = FP64 copies of the mixed state)
    and the backward recomputes each segment in FP64. Its force history is
    the mixed step's, and its gradients follow the FP64-forward adjoint's to
    the distance between the two trajectories."""
    from icempm_3dm_b200 import PRECISION_MIXED
    prms, soa, coh = case(n=3000, seed=11)
    n = soa.shape[1]
    nsteps, every = 40, 10
    rng = np.random.default_rng(3)
    wgt = rng.standard_normal((nsteps, 3))
    wgt[:, 2] = 0.0
    out = {}
    for prec in (PRECISION_FP64_SVD64, PRECISION_MIXED):
        with MPMHandle(prms, n, prec) as h:
            h.upload(soa, cohesion=coh)
            hist = np.zeros((nsteps, 3))
            check(LIB.mpm_adjoint_forward(h._h, nsteps, every, dptr(hist)), "adjoint forward")
            dc = np.zeros(n)
            dE = ctypes.c_double(0)
            check(LIB.mpm_adjoint_backward(h._h, dptr(np.ascontiguousarray(wgt)), dptr(dc), ctypes.byref(dE)),
                  "adjoint backward")
            out[prec] = (hist, dc, dE.value)
        with MPMHandle(prms, n, prec) as h:
            h.upload(soa, cohesion=coh)
            ref = h.step(nsteps)
        assert np.linalg.norm(out[prec][0] - ref) <= 1e-6 * np.linalg.norm(ref), prec
    (h64, dc64, dE64), (hmx, dcmx, dEmx) = out[PRECISION_FP64_SVD64], out[PRECISION_MIXED]
    e_hist = np.linalg.norm(hmx - h64) / np.linalg.norm(h64)
    e_c = np.abs(dcmx - dc64).max() / np.abs(dc64).max()
    e_E = abs(dEmx - dE64) / abs(dE64)
    print(f"\nmixed vs FP64 forward: force history {e_hist:.2e}; dL/dc {e_c:.2e} of the largest; dL/dE {e_E:.2e}")
    assert np.count_nonzero(dcmx) > n // 2
    assert e_hist < 1e-3 and e_c < 1e-2 and e_E < 1e-2
