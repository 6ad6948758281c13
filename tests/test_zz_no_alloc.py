"""The allocation-free sort entry point (mpm_sort_permutation_noalloc), for
callers that manage all device memory themselves or cannot stop for a
cudaMalloc mid-run. The caller owns the input and output buffers (here torch
CUDA tensors); the library's scratch is its fixed array. Calls in a row, on
different inputs and grids, must give exactly the permutation of the existing
entry point mpm_sort (integer results: bit-exact), so each later call also
shows that what the earlier one left in the shared array does not leak into
it: a smaller grid with halo slabs after a larger one, a valid call after
one that stopped on a particle outside the grid, a row pitch above the
particle count, and no particles at all.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import LIB
from icempm_3dm_b200.layout import IDX_UTILITY, POSX, STATUS_DISABLED
from tests.helpers import perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.gpu


def shuffled(prms, soa, seed, disabled_frac):
    n = soa.shape[1]
    rng = np.random.default_rng(seed)
    soa = np.ascontiguousarray(soa[:, rng.permutation(n)])
    bits = util_bits(soa).copy()
    bits[rng.random(n) < disabled_frac] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    soa[POSX:POSX + 3, 1:100:2] = soa[POSX:POSX + 3, 0:99:2]     # ties keep their order
    return prms, soa


def shuffled_block(n, seed, disabled_frac):
    prms, soa = perturbed_block(n=n, seed=seed)
    return shuffled(prms, soa, seed, disabled_frac)


def noalloc_sort(prms, soa, n=None, expect=0):
    """Calls the entry point on device copies of soa (its full width is the
    row pitch; the first n columns are the particles). Returns the kept
    permutation, or None when expect != 0."""
    import torch
    pitch = soa.shape[1]
    n = pitch if n is None else n
    d_soa = torch.from_numpy(np.ascontiguousarray(soa)).cuda()
    d_perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    kept = ctypes.c_uint(12345)
    stream = torch.cuda.current_stream().cuda_stream
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(prms), ctypes.c_void_p(d_soa.data_ptr()), pitch, n,
                                          ctypes.c_void_p(d_perm.data_ptr()), ctypes.byref(kept),
                                          ctypes.c_void_p(stream))
    assert rc == expect, rc
    if expect:
        return None
    return d_perm[:kept.value].cpu().numpy().view(np.uint32)


def sort_with_handle(prms, soa):
    with MPMHandle(prms, soa.shape[1]) as h:
        h.upload(soa)
        assert h.sort() == 0
        return h.ids()


def test_calls_in_a_row_match_mpm_sort():
    big = shuffled_block(20000, 91, 0.05)
    p_small, s_small, _ = gen.small_block(n=6000, seed=92, dims=(0.12, 0.08, 0.08), halo=3)
    small = shuffled(p_small, s_small, 92, 0.2)
    assert small[0].GridHaloSize == 3
    assert small[0].GridXTotal * small[0].GridY * small[0].GridZ < big[0].GridXTotal * big[0].GridY * big[0].GridZ
    for prms, soa in (big, small, big):
        got = noalloc_sort(prms, soa)
        ref = sort_with_handle(prms, soa)
        assert got.shape == ref.shape
        assert np.array_equal(got, ref)


def test_out_of_grid_stops_then_the_next_call_sorts():
    prms, soa = shuffled_block(5000, 93, 0.05)
    bad = soa.copy()
    bad[POSX, 17] = -5.0                 # far outside the grid in -x
    noalloc_sort(prms, bad, expect=107)
    with MPMHandle(prms, soa.shape[1]) as h:
        h.upload(bad)
        assert LIB.mpm_sort(h._h) == 107     # the existing entry point refuses it the same way
    got = noalloc_sort(prms, soa)
    assert np.array_equal(got, sort_with_handle(prms, soa))


def test_pitch_above_n_and_no_particles():
    prms, soa = shuffled_block(3000, 94, 0.1)
    n = soa.shape[1]
    wide = np.zeros((soa.shape[0], n + 37))
    wide[:, :n] = soa
    wide[POSX:POSX + 3, n:] = 1e9         # columns past n are not particles and must not be read as such
    got = noalloc_sort(prms, wide, n=n)
    assert np.array_equal(got, sort_with_handle(prms, soa))
    assert noalloc_sort(prms, soa, n=0).size == 0


def test_sizes_beyond_the_fixed_scratch_are_rejected():
    """Rejected before any device work, with real (small) device buffers."""
    import torch
    prms, soa = shuffled_block(4000, 95, 0.0)
    d_soa = torch.from_numpy(soa).cuda()
    d_perm = torch.zeros(soa.shape[1], dtype=torch.int32, device="cuda")
    kept = ctypes.c_uint(0)
    big = prms.copy()
    big.GridXTotal = 4000          # far more cell keys than the scratch holds
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(big), ctypes.c_void_p(d_soa.data_ptr()), soa.shape[1],
                                          soa.shape[1], ctypes.c_void_p(d_perm.data_ptr()), ctypes.byref(kept), None)
    assert rc == 109
    d_many = torch.zeros((28, (1 << 19) + 1), dtype=torch.float64, device="cuda")
    d_perm_many = torch.zeros((1 << 19) + 1, dtype=torch.int32, device="cuda")
    n_many = (1 << 19) + 1         # one particle more than the scratch holds
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(prms), ctypes.c_void_p(d_many.data_ptr()), n_many, n_many,
                                          ctypes.c_void_p(d_perm_many.data_ptr()), ctypes.byref(kept), None)
    assert rc == 109
    # a valid call afterwards still works
    assert np.array_equal(noalloc_sort(prms, soa), sort_with_handle(prms, soa))
