"""Page-locked host arrays (icempm_3dm_b200.pinned_empty over mpm_host_alloc /
mpm_host_free): the memory outlives every view of it and is released exactly
once. On CPU the two library calls are replaced by fakes over ordinary
memory; tests/test_gpu_host_memory.py uses the real ones."""
import ctypes
import gc

import numpy as np

from icempm_3dm_b200 import simulation
from icempm_3dm_b200._lib import LIB


def test_pinned_array_lives_as_long_as_its_views(monkeypatch):
    blocks, freed = {}, []

    def fake_alloc(nbytes, out):
        buf = ctypes.create_string_buffer(nbytes)
        blocks[ctypes.addressof(buf)] = buf
        out._obj.value = ctypes.addressof(buf)
        return 0

    def fake_free(ptr):
        freed.append(ptr.value)
        return 0

    monkeypatch.setattr(LIB, "mpm_host_alloc", fake_alloc)
    monkeypatch.setattr(LIB, "mpm_host_free", fake_free)
    a = simulation.pinned_empty((28, 100))
    assert a.shape == (28, 100) and a.dtype == np.float64 and a.flags.c_contiguous
    addr = a.ctypes.data
    assert addr in blocks
    a[:] = np.arange(2800.0).reshape(28, 100)
    view = a[:, :10]
    del a
    gc.collect()
    assert freed == []                       # the view keeps the memory
    assert view[27, 9] == 2709.0
    del view
    gc.collect()
    assert freed == [addr]                   # released once, with the last view
    assert simulation.pinned_empty((0, 5)).size == 0 and len(blocks) == 1
