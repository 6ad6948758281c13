"""Edge cases of the step API on the GPU, both precisions: empty inputs,
every particle disabled, uploads beyond the capacity, and particle counts
that leave partial warps and blocks (1, 33, 1001) against the oracle."""
import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_MIXED
from icempm_3dm_b200._lib import BP00, IDX_JP_INV, IDX_UTILITY, LIB, POSX, STATUS_DISABLED, dptr
from oracle import pyoracle as po
from tests.helpers import perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.gpu

PRECISIONS = [PRECISION_FP64, PRECISION_MIXED]
STATE_ROWS = list(range(POSX, BP00 + 9)) + [IDX_JP_INV]


@pytest.mark.parametrize("precision", PRECISIONS)
def test_empty_upload_steps_sorts_and_downloads(precision):
    prms, soa = perturbed_block(n=500, seed=3)
    with MPMHandle(prms, 500, precision) as h:
        h.upload(np.ascontiguousarray(soa[:, :0]))
        assert h.count() == 0
        hist = h.step(4)
        assert np.all(hist == 0)
        assert h.sort() == 0
        assert h.count() == 0
        assert h.download().shape == (soa.shape[0], 0)
        assert h.ids().size == 0
        assert h.params().SimulationStep == 4


@pytest.mark.parametrize("precision", PRECISIONS)
def test_sort_with_every_particle_disabled_leaves_none(precision):
    prms, soa = perturbed_block(n=700, seed=4)
    bits = util_bits(soa) | STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    with MPMHandle(prms, soa.shape[1], precision) as h:
        h.upload(soa)
        h.step(2)
        assert h.sort() == 0
        assert h.count() == 0
        assert np.all(h.step(3) == 0)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_upload_beyond_capacity_is_refused_and_handle_stays_usable(precision):
    prms, soa = perturbed_block(n=600, seed=5)
    n = soa.shape[1]
    with MPMHandle(prms, n - 100, precision) as h:
        assert LIB.mpm_upload_soa(h._h, dptr(soa), n, n) == 102
        part = np.ascontiguousarray(soa[:, :n - 100])
        h.upload(part)
        assert h.count() == n - 100
        h.step(2)
        assert h.download().shape == part.shape


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("n", [1, 33, 1001])
def test_partial_warps_and_blocks_match_oracle(n, precision):
    prms, soa = perturbed_block(n=3000, seed=9, ind_velocity=0.5, crushed_frac=0.1)
    soa = np.ascontiguousarray(soa[:, :n])
    steps = 20
    with MPMHandle(prms, n, precision) as h:
        h.upload(soa)
        hist = h.step(steps)
        out = h.download()
    sim = po.OracleSim(prms, soa, n, svd_mode=0 if precision == PRECISION_FP64 else 1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    assert out.shape == sim.soa.shape
    norm = float(np.linalg.norm(ref_hist))
    if precision == PRECISION_FP64:
        assert np.abs(hist - ref_hist).max() <= 1e-7 * max(np.abs(ref_hist).max(), 1e-300) + 1e-9
        assert np.array_equal(util_bits(out), util_bits(sim.soa))
        for r in STATE_ROWS:
            scale = max(np.abs(sim.soa[r]).max(), 1e-300)
            assert np.abs(out[r] - sim.soa[r]).max() <= 1e-7 * scale + 1e-10, r
    else:
        if norm > 0:
            assert np.linalg.norm(hist - ref_hist) / norm < 1e-3
        else:
            assert np.abs(hist).max() < 1e-6
        assert np.abs(out[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < 1e-6


@pytest.mark.parametrize("precision", PRECISIONS)
def test_frame_records_of_empty_and_fully_disabled_inputs(precision):
    """mpm_frame_records with no particles, or with every particle disabled:
    the scans run over a single sentinel element and no record comes out."""
    prms, soa = perturbed_block(n=300, seed=6)
    with MPMHandle(prms, 300, precision) as h:
        h.upload(np.ascontiguousarray(soa[:, :0]))
        assert h.frame_records(0, True).size == 0
        assert all(r.size == 0 for r in h.frame_records(1, False))
        bits = util_bits(soa) | STATUS_DISABLED
        soa[IDX_UTILITY] = util_as_double(bits)
        h.upload(soa)
        with pytest.raises(Exception):
            h.frame_records(2, False)           # an upload asks for a full frame first
        assert h.frame_records(2, True).size == 0
        h.step(2)
        assert all(r.size == 0 for r in h.frame_records(3, False))
