"""The CUDA path against the reference's own kernels.

tests/golden/ref_steps.npz holds runs of simulation/mpm_kernels.cuh itself
(compiled as host C++ from the reference tree, oracle/ref_kernels.cpp; made by
tests/golden/make_ref_fixtures.py): three seeded inputs, 20 substeps each, the
input state, the force history and the final state. Here the same inputs go
through the C-ABI:

  FP64 mode (the reference's arithmetic, FP32 SVD): force history within
  1e-8 and every state field within 1e-8 of its largest magnitude (the GPU
  contracts products into fused multiply-adds and sums the P2G atomics in
  another order, the reference build here does neither); status words (the
  crushed flags) bit for bit.
  mixed mode: force history within 1e-3 (the mixed path's bound), positions
  within 1e-6 m.

For liquid particles the reference stores trial P and Q it never computed
(mpm_kernels.cuh:316-327,347-351); those entries are not compared.
"""
import os

import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_MIXED, SimParams3D
from icempm_3dm_b200.layout import POSX, STATUS_LIQUID
from tests.helpers import util_bits

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_steps.npz")
CASES = ("crushed", "liquid", "halo")
FIELDS = (("Jp_inv", 3, 4), ("x", 4, 7), ("v", 7, 10), ("F", 10, 19), ("C", 19, 28))


def load(name):
    z = np.load(GOLDEN)
    prms = SimParams3D.from_buffer_copy(z[f"{name}_params"].tobytes())
    return prms, z[f"{name}_soa"], z[f"{name}_hist"], z[f"{name}_out"], int(z["steps"])


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_the_reference_kernels(name):
    prms, soa, hist, out, steps = load(name)
    n = soa.shape[1]
    with MPMHandle(prms, n, PRECISION_FP64) as h:
        h.upload(soa)
        got_hist = h.step(steps)
        got = h.download()
    e = float(np.linalg.norm(got_hist - hist) / np.linalg.norm(hist))
    assert np.linalg.norm(hist) > 0
    assert e < 1e-8, e
    assert np.array_equal(util_bits(got), util_bits(out))
    errs = {f: rel(got[a:b], out[a:b]) for f, a, b in FIELDS}
    solid = (util_bits(out) & STATUS_LIQUID) == 0
    errs["P, Q"] = rel(got[1:3, solid], out[1:3, solid])
    print(f"\n{name}: force {e:.2e}, " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v < 1e-8, k


@pytest.mark.parametrize("name", CASES)
def test_mixed_force_history_within_bound_of_the_reference(name):
    prms, soa, hist, out, steps = load(name)
    n = soa.shape[1]
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.upload(soa)
        got_hist = h.step(steps)
        got = h.download()
    e = float(np.linalg.norm(got_hist - hist) / np.linalg.norm(hist))
    x = float(np.abs(got[POSX:POSX + 3] - out[POSX:POSX + 3]).max())
    print(f"\n{name} mixed: force {e:.2e}, positions {x:.2e} m")
    assert e < 1e-3
    assert x < 1e-6
