"""Downloads into page-locked host memory (pinned_empty, mpm_host_alloc) give
the same particles as into ordinary memory, and the Model3D mirror's
transfer_from_device reuses one such buffer from frame to frame."""
import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, Model3D, PRECISION_FP64, PRECISION_MIXED, pinned_empty
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200.layout import N_PTS_ARRAYS

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED], ids=["fp64", "mixed"])
def test_pinned_download_equals_plain_download(precision):
    prms, soa, _ = gen.small_block(n=6000, seed=91)
    n = soa.shape[1]
    with MPMHandle(prms, n + 17, precision) as h:
        host = pinned_empty((N_PTS_ARRAYS, h.capacity))
        h.upload(soa)
        h.step(5)
        plain = h.download()
        pinned = h.download(out=host)
        assert pinned.shape == plain.shape
        assert np.array_equal(pinned.view(np.int64), plain.view(np.int64))
        assert pinned.ctypes.data == host.ctypes.data
        h.upload(np.ascontiguousarray(pinned))          # and back up from page-locked memory
        assert np.array_equal(h.download().view(np.int64), plain.view(np.int64))
        with pytest.raises(ValueError):
            h.download(out=np.zeros((N_PTS_ARRAYS, 3)))


def test_model_transfer_reuses_one_host_buffer():
    prms, soa, _ = gen.small_block(n=4000, seed=92)
    prms.UpdateEveryNthStep = 5
    model = Model3D(prms, soa)
    model.Step()
    first = model.gpu.hssoa.ctypes.data
    after_one = model.gpu.hssoa.copy()
    model.Step()
    assert model.gpu.hssoa.ctypes.data == first
    assert np.array_equal(model.gpu.hssoa.view(np.int64), model.gpu.handle.download().view(np.int64))
    assert not np.array_equal(model.gpu.hssoa, after_one)
