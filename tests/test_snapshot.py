"""SnapshotManager mirror on CPU: LoadRawPoints placement on the reference's
own input (input_data/p1.json + build/geometries_3d/3d_200k.h5), the full
snapshot d%05d.h5 written and read back, and ReadParametersFromAttributes'
behaviour (DP_threshold_p is not restored)."""
import ctypes
import math
import os

import numpy as np
import pytest

from icempm_3dm_b200 import SimParams3D, snapshot
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import FE00, IDX_JP_INV, IDX_UTILITY, LIB, N_PTS_ARRAYS, POSX
from icempm_3dm_b200.h5io import H5File

from oracle import pyoracle as po  # noqa: E402

REF = po.reference_tree() or ""          # the tree oracle/_ref was built from, if on this machine
P1 = os.path.join(REF, "input_data", "p1.json")
PC = os.path.join(REF, "build", "geometries_3d", "3d_200k.h5")
needs_ref = pytest.mark.skipif(not (os.path.exists(P1) and os.path.exists(PC)), reason="reference inputs not present")


def parse(path):
    p = SimParams3D()
    raw = ctypes.create_string_buffer(4096)
    assert LIB.mpm_params_parse_file(p, path.encode(), raw, len(raw)) == 0
    return p, raw.value.decode()


@needs_ref
def test_load_raw_points_places_the_reference_block_as_load_raw_points_does():
    p, raw = parse(P1)
    assert raw == "geometries_3d/3d_200k.h5"
    q, soa, cap = snapshot.load_raw_points(PC, p)
    n = 202329
    assert soa.shape == (N_PTS_ARRAYS, n) and q.nPtsTotal == n
    assert cap == int(n * (1 + p.ExtraSpaceForIncomingPoints))
    with H5File(PC) as f:
        g = f.read("llGrainIDs")
        raw_pos = np.stack([f.read(k) for k in "xyz"])
    assert np.array_equal(soa[IDX_UTILITY].view(np.uint64), g)
    h = q.cellsize
    pos = soa[POSX:POSX + 3]
    lo, hi = raw_pos.min(axis=1), raw_pos.max(axis=1)
    assert (q.xmin, q.ymin, q.zmin, q.xmax, q.ymax, q.zmax) == (*lo, *hi)
    # snapshotmanager.cpp:57-64: x and z shifted by (box - length) / 2, y so
    # that the lowest point is 2h above the floor
    x_off = (q.GridXTotal * h - (hi[0] - lo[0])) / 2
    off = np.array([x_off, 2 * h - lo[1], (q.GridZ * h - (hi[2] - lo[2])) / 2])
    assert np.array_equal(pos, raw_pos + off[:, None])
    assert np.all(soa[IDX_JP_INV] == 1.0)
    for r in range(3):
        for c in range(3):
            assert np.all(soa[FE00 + 3 * r + c] == (1.0 if r == c else 0.0))
    assert q.Volume == 3.75 and q.ParticleVolume == 3.75 / n
    r = q.IndDiameter / 2
    ht = r - q.IndDepth
    assert q.indenter_x == math.floor((x_off - math.sqrt(r * r - ht * ht)) / h) * h
    assert q.indenter_y == q.ymax + (2 * h - q.ymin) + ht
    assert (q.indenter_x_initial, q.indenter_y_initial) == (q.indenter_x, q.indenter_y)


def _params():
    p = gen.make_params(gen.CONFIGS["block250k"], 1000)
    p.SimulationStep, p.SimulationTime = 375, 375 * p.InitialTimeStep
    p.indenter_x += 0.0123
    p.DP_threshold_p = 12345.0
    return p


@pytest.mark.parametrize("compress", [False, True])
def test_snapshot_round_trip(tmp_path, compress):
    p = _params()
    rng = np.random.default_rng(1)
    cap, size = 1500, 1000
    hs = np.zeros((N_PTS_ARRAYS, cap))
    hs[:, :size] = rng.standard_normal((N_PTS_ARRAYS, size))
    ind = rng.standard_normal(3 * p.IndenterSubdivisions * p.GridZ)
    path = snapshot.save_snapshot(str(tmp_path / "snaps"), snapshot.animation_frame_number(p), p, hs, size, ind,
                                  compress=compress)
    assert os.path.basename(path) == "d%05d.h5" % (375 // p.UpdateEveryNthStep)
    with H5File(path) as f:
        assert f.keys() == ["Indenter", "Points"]
        a = f.attrs("Points")
        assert list(a)[:2] == ["HSSOA_capacity", "HSSOA_size"]
        assert [k for k in a][2:] == [k for k, _ in snapshot.PARAM_ATTRS]
        assert a["HSSOA_capacity"].dtype == np.uint32 and a["GridY"].dtype == np.int32
        assert f.shape("Points") == (cap * N_PTS_ARRAYS,)
    q, hs2, size2, ind2 = snapshot.read_snapshot(path)
    assert size2 == size and np.array_equal(hs2, hs) and np.array_equal(ind2, ind)
    for name, _ in snapshot.PARAM_ATTRS:
        if name == "DP_threshold_p":
            continue
        assert getattr(q, name) == getattr(p, name), name
    for derived in ("mu", "kappa", "lambda_", "cellsize_inv", "dt_vol_Dpinv", "ParticleMass", "IndRSq"):
        assert getattr(q, derived) == pytest.approx(getattr(p, derived), rel=1e-15), derived


def test_read_parameters_from_attributes_does_not_restore_dp_threshold(tmp_path):
    p = _params()
    d = SimParams3D()
    LIB.mpm_params_reset(d)
    assert d.DP_threshold_p != p.DP_threshold_p
    q = snapshot.params_from_attributes(snapshot.params_as_attributes(p))
    assert q.DP_threshold_p == d.DP_threshold_p
    attrs = snapshot.params_as_attributes(p)
    del attrs["animation_threshold_pos"]
    assert snapshot.params_from_attributes(attrs).animation_threshold_pos == d.animation_threshold_pos
    del attrs["GridY"]
    with pytest.raises(KeyError):
        snapshot.params_from_attributes(attrs)


def test_partitions_override_and_missing_files(tmp_path):
    p = _params()
    hs = np.zeros((N_PTS_ARRAYS, 10))
    path = snapshot.save_snapshot(str(tmp_path), 0, p, hs, 10, np.zeros(3 * p.IndenterSubdivisions * p.GridZ))
    q, *_ = snapshot.read_snapshot(path, partitions=3)
    assert q.nPartitions == 3
    with pytest.raises(FileNotFoundError):
        snapshot.read_snapshot(str(tmp_path / "nope.h5"))
    with pytest.raises(FileNotFoundError):
        snapshot.load_raw_points(str(tmp_path / "nope.h5"), p)
    with pytest.raises(ValueError):
        snapshot.save_snapshot(str(tmp_path), 1, p, hs, 10, np.zeros(5))


def test_frame_file_layout(tmp_path):
    """SaveFrame's file: Indenter (chunks of min(10000, size), deflate 5) with
    its attributes in order, VisualPoints or the non-empty delta datasets as
    compounds with the reference's member names, offsets and sizes."""
    from icempm_3dm_b200 import h5io
    p = _params()
    ind = np.arange(3 * p.IndenterSubdivisions * p.GridZ, dtype=np.float64)
    pts = np.zeros(50, dtype=snapshot.VISUAL_POINT)
    pts["px"] = np.arange(50)
    pts["status"] = 0x83
    full = snapshot.save_frame(str(tmp_path), 7, p, ind, [1.0, 2.0, 3.0], False, points=pts, timestamp=1234)
    pv = np.zeros(4, dtype=snapshot.UPDATE_POS)
    pv["idx"] = [1, 5, 9, 11]
    jp = np.zeros(0, dtype=snapshot.UPDATE_JP)
    st = np.zeros(2, dtype=snapshot.UPDATE_STATUS)
    st["status"] = [0x80, 0x01]
    part = snapshot.save_frame(str(tmp_path), 8, p, ind, [0.0, 0.0, 0.0], True, upd_pos=pv, upd_jp=jp, upd_status=st)
    assert full.endswith("v00007.h5") and part.endswith("v00008.h5")
    f = snapshot.read_frame(full)
    assert list(f["attrs"])[:4] == ["indenter_total_x", "indenter_total_y", "indenter_total_z", "partial_frame"]
    assert list(f["attrs"])[-1] == "timestamp" and f["attrs"]["timestamp"] == 1234
    assert f["attrs"]["timestamp"].dtype == np.uint64 and f["attrs"]["partial_frame"].dtype == np.uint8
    assert f["attrs"]["indenter_total_z"] == 3.0 and f["attrs"]["partial_frame"] == 0
    assert np.array_equal(f["Indenter"], ind) and np.array_equal(f["VisualPoints"], pts)
    g = snapshot.read_frame(part)
    assert g["attrs"]["partial_frame"] == 1
    assert set(g) == {"attrs", "Indenter", "UpdatePos", "UpdateStatus"}      # empty UpdateJp is not written
    assert np.array_equal(g["UpdatePos"], pv) and np.array_equal(g["UpdateStatus"], st)
    assert snapshot.UPDATE_POS.itemsize == 28 and snapshot.UPDATE_STATUS.itemsize == 8
    with h5io.H5File(full) as h:
        lay = [h5io._parse_layout(d) for t, fl, d in h._messages(h._datasets["Indenter"]) if t == 0x08][0]
        filt = [h5io._parse_filters(d) for t, fl, d in h._messages(h._datasets["VisualPoints"]) if t == 0x0B][0]
    assert lay[0] == "chunked" and lay[2] == (min(10000, ind.size), 8)
    assert filt == [(1, 1, (5,))]
