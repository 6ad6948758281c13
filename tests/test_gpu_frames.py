"""mpm_frame_records (SnapshotManager::SaveFrame's records, built on the
device) against the float32 CPU restatement in oracle/frames.py, bit for bit:
a full frame, then partial frames carrying the refresh state; disabled
points shift the visual index, partition bits and the crushed flag form the
status byte. Then Model3D + SnapshotManager.SaveFrame write v%05d.h5 files."""
import numpy as np
import pytest

from icempm_3dm_b200 import PRECISION_FP64, PRECISION_MIXED, MPMHandle, Model3D, SnapshotManager, snapshot
from icempm_3dm_b200._lib import IDX_UTILITY, STATUS_DISABLED
from oracle import frames as of
from tests.helpers import perturbed_block, util_as_double, util_bits

pytestmark = pytest.mark.gpu


def block(seed=5):
    prms, soa = perturbed_block(n=4000, seed=seed, crushed_frac=0.1, strong_frac=0.2, ind_velocity=0.5)
    rng = np.random.default_rng(seed)
    bits = util_bits(soa)
    bits[rng.random(soa.shape[1]) < 0.03] |= STATUS_DISABLED
    bits[rng.random(soa.shape[1]) < 0.3] |= np.int64(3) << 24          # a partition id in bits 24-31
    soa[IDX_UTILITY] = util_as_double(bits)
    prms.animation_threshold_pos = 2e-6
    return prms, soa


def same_visual(rec, pos, vel, jp, status):
    assert rec.size == pos.shape[1]
    for d, k in enumerate(("px", "py", "pz")):
        assert np.array_equal(rec[k], pos[d])
    for d, k in enumerate(("vx", "vy", "vz")):
        assert np.array_equal(rec[k], vel[d])
    assert np.array_equal(rec["Jp_inv"], jp) and np.array_equal(rec["status"], status)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_frame_records_match_the_cpu_restatement(precision):
    prms, soa = block()
    n = soa.shape[1]
    st = of.FrameState()
    with MPMHandle(prms, n, precision) as h:
        h.upload(soa)
        with pytest.raises(Exception):
            h.frame_records(0, False)                   # no full frame yet: MPM_ERR_STATE
        full = h.frame_records(0, True)
        same_visual(full, *st.full(h.download(), 0))
        assert full.size == int((util_bits(soa) & STATUS_DISABLED == 0).sum())
        assert set(np.unique(full["status"] & 0x7F)) <= {0, 3}
        totals = np.zeros(3, dtype=np.int64)
        for frame in (1, 2, 3):
            h.step(15)
            pv, jp, stt = h.frame_records(frame, False)
            (ipv, ijp, ist), (pos, vel, jpv, sts) = st.partial(h.download(), frame, prms.InitialTimeStep,
                                                               prms.UpdateEveryNthStep, prms.animation_threshold_pos)
            assert np.array_equal(pv["idx"], ipv) and np.array_equal(jp["idx"], ijp) and np.array_equal(stt["idx"], ist)
            for d, k in enumerate(("px", "py", "pz")):
                assert np.array_equal(pv[k], pos[d, ipv])
            for d, k in enumerate(("vx", "vy", "vz")):
                assert np.array_equal(pv[k], vel[d, ipv])
            assert np.array_equal(jp["Jp_inv"], jpv[ijp]) and np.array_equal(stt["status"], sts[ist])
            totals += (pv.size, jp.size, stt.size)
        assert totals[0] > 0 and totals[2] > 0, totals     # refreshes and newly crushed points occur


def test_model_save_frame_writes_full_then_partial_frames(tmp_path):
    prms, soa = block(seed=8)
    model = Model3D(prms, soa)
    sm = SnapshotManager(model)
    model.Step(substeps=10)
    p0 = sm.SaveFrame(str(tmp_path), 1)
    model.Step(substeps=10)
    p1 = sm.SaveFrame(str(tmp_path), 2)
    f0, f1 = snapshot.read_frame(p0), snapshot.read_frame(p1)
    assert p0.endswith("v00001.h5") and p1.endswith("v00002.h5")
    assert f0["attrs"]["partial_frame"] == 0 and f1["attrs"]["partial_frame"] == 1
    assert "VisualPoints" in f0 and "VisualPoints" not in f1
    assert f0["VisualPoints"].dtype == snapshot.VISUAL_POINT
    assert f0["VisualPoints"].size == model.gpu.hssoa.shape[1] - int(
        (util_bits(model.gpu.hssoa) & STATUS_DISABLED != 0).sum())
    assert "UpdatePos" in f1 and f1["UpdatePos"].dtype == snapshot.UPDATE_POS
    assert np.array_equal(f1["Indenter"], model.gpu.indenter_sensor_total)
    assert f1["attrs"]["indenter_total_x"] == model.gpu.indenter_force[0]
    assert f1["attrs"]["SimulationStep"] == 20
