"""The allocation-free sort entry point (mpm_sort_permutation_noalloc), for
callers that manage all device memory themselves or cannot stop for a
cudaMalloc mid-run. The caller owns the input and output buffers (here torch
CUDA tensors); the library's scratch is its fixed array. Two calls in a row,
on different inputs, must give exactly the permutation of the existing
entry point mpm_sort (integer results: bit-exact), so the second call also
shows that what the first left in the shared array does not leak into it.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle
from icempm_3dm_b200._lib import IDX_UTILITY, LIB, POSX, STATUS_DISABLED
from tests.helpers import perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.gpu


def shuffled_block(n, seed, disabled_frac):
    prms, soa = perturbed_block(n=n, seed=seed)
    n = soa.shape[1]
    rng = np.random.default_rng(seed)
    soa = np.ascontiguousarray(soa[:, rng.permutation(n)])
    bits = util_bits(soa).copy()
    bits[rng.random(n) < disabled_frac] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    soa[POSX:POSX + 3, 1:100:2] = soa[POSX:POSX + 3, 0:99:2]     # ties keep their order
    return prms, soa


def noalloc_sort(prms, soa):
    import torch
    n = soa.shape[1]
    d_soa = torch.from_numpy(soa).cuda()
    d_perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    kept = ctypes.c_uint(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(prms), ctypes.c_void_p(d_soa.data_ptr()), n, n,
                                          ctypes.c_void_p(d_perm.data_ptr()), ctypes.byref(kept),
                                          ctypes.c_void_p(stream))
    assert rc == 0, rc
    return d_perm[:kept.value].cpu().numpy().view(np.uint32)


def sort_with_handle(prms, soa):
    with MPMHandle(prms, soa.shape[1]) as h:
        h.upload(soa)
        assert h.sort() == 0
        return h.ids()


def test_two_calls_match_mpm_sort():
    for seed, n, frac in ((91, 20000, 0.05), (92, 12000, 0.2)):
        prms, soa = shuffled_block(n, seed, frac)
        got = noalloc_sort(prms, soa)
        ref = sort_with_handle(prms, soa)
        assert got.shape == ref.shape
        assert np.array_equal(got, ref)


def test_sizes_beyond_the_fixed_scratch_are_rejected():
    prms, soa = shuffled_block(4000, 93, 0.0)
    kept = ctypes.c_uint(0)
    big = prms.copy()
    big.GridXTotal = 4000          # far more cell keys than the scratch holds
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(big), ctypes.c_void_p(1), 4000, 4000, ctypes.c_void_p(1),
                                          ctypes.byref(kept), None)
    assert rc == 109
    rc = LIB.mpm_sort_permutation_noalloc(ctypes.byref(prms), ctypes.c_void_p(1), 1 << 20, 1 << 20,
                                          ctypes.c_void_p(1), ctypes.byref(kept), None)
    assert rc == 109
