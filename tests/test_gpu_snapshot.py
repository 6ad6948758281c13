"""The reference's input and checkpoint path on the GPU: a JSON configuration
with the reference's keys and a point cloud in the reference's raw-point HDF5
layout (llGrainIDs, x, y, z, 'volume'; chunked, deflate) go through
Model3D.from_config (ParseFile + LoadRawPoints + device sort) and step against
the oracle; SaveSnapshot -> ReadSnapshot -> Step continues a run as if it had
not been interrupted."""
import ctypes
import json

import numpy as np
import pytest

from icempm_3dm_b200 import (LIB, PRECISION_FP64, PRECISION_MIXED, Model3D, SimParams3D, SnapshotManager,
                             snapshot)
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import POSX, STATUS_LIQUID, VELX
from icempm_3dm_b200.h5io import H5Writer
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

DIMS = (0.4, 0.15, 0.2)


def write_case(tmp, n=20000, seed=7, **extra):
    """pc.h5 + case.json in tmp; DP_threshold_p is the Reset() value (the
    one ReadSnapshot leaves in place); extra JSON keys override."""
    pos = gen.jittered_lattice(n, DIMS, seed)
    grains = np.floor(gen.uniform(seed, np.arange(n), 3) * 100).astype(np.uint64)
    with H5Writer(tmp / "pc.h5") as w:
        w.create_dataset("llGrainIDs", grains, chunks=(8192,), deflate=7,
                         attrs={"volume": np.float64(np.prod(DIMS))})
        for d, k in enumerate("xyz"):
            w.create_dataset(k, pos[d], chunks=(8192,), deflate=7)
    d = SimParams3D()
    LIB.mpm_params_reset(d)
    cfg = {"InputRawPoints": "pc.h5", "nPartitions": 1, "GridHaloSize": 0, "ExtraSpaceForIncomingPoints": 0.2,
           "InitialTimeStep": 1e-5, "GridX": 80, "GridY": 30, "GridZ": 40, "DomainDimensionX": 0.8,
           "YoungsModulus": 5e8, "IceCompressiveStrength": 100e6, "IceTensileStrength": 10e6,
           "IceTensileStrength2": 10e6, "IceShearStrength": 7e6, "DP_phi": 62, "DP_threshold_p": d.DP_threshold_p,
           "SimulationEndTime": 1.0, "PoissonsRatio": 0.3, "Gravity": 9.81, "Density": 917,
           "IndDiameter": 0.1, "IndVelocity": 1.0, "IndDepth": 0.05}
    cfg.update(extra)
    (tmp / "case.json").write_text(json.dumps(cfg))
    return tmp / "case.json"


def parsed(js):
    p = SimParams3D()
    raw = ctypes.create_string_buffer(256)
    assert LIB.mpm_params_parse_file(p, str(js).encode(), raw, 256) == 0
    return p


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_config_and_point_cloud_through_the_gpu_step(tmp_path, precision):
    js = write_case(tmp_path)
    model = Model3D.from_config(js, base_dir=tmp_path, precision=precision)
    p = model.prms
    q, soa, cap = snapshot.load_raw_points(str(tmp_path / "pc.h5"), parsed(js))
    n = soa.shape[1]
    perm = po.sort_permutation(q, soa, n)
    ref0 = np.ascontiguousarray(soa[:, perm])
    assert model.gpu.handle.capacity == cap
    assert np.array_equal(model.gpu.handle.ids(), perm)
    held = model.gpu.hssoa
    if precision == PRECISION_FP64:
        assert np.array_equal(held, ref0)
    else:
        assert np.abs(held[POSX:POSX + 3] - ref0[POSX:POSX + 3]).max() < 2e-8
    assert (p.SimulationStep, p.SimulationTime) == (0, 0.0)
    steps = 40
    hist = model.gpu.handle.step(steps)
    sim = po.OracleSim(p, ref0, n, svd_mode=0 if precision == PRECISION_FP64 else 1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    norm = float(np.linalg.norm(ref_hist))
    assert norm > 0, "the indenter should touch the block"
    e = float(np.linalg.norm(hist - ref_hist)) / norm
    assert e < (1e-7 if precision == PRECISION_FP64 else 1e-3), e
    out = model.gpu.handle.download()
    assert np.abs(out[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < (1e-10 if precision == PRECISION_FP64 else 1e-6)


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
@pytest.mark.parametrize("compress", [False, True])
def test_snapshot_resume_matches_the_uninterrupted_run(tmp_path, precision, compress):
    js = write_case(tmp_path)
    a = Model3D.from_config(js, base_dir=tmp_path, precision=precision)
    a.Step(substeps=25)
    path = SnapshotManager(a).SaveSnapshot(str(tmp_path / "snaps"), snapshot.animation_frame_number(a.prms),
                                           compress)
    a.Step(substeps=25)
    out_a = a.gpu.hssoa
    b = Model3D.from_snapshot(path, precision=precision)
    assert b.prms.SimulationStep == 25 and b.prms.SimulationTime == pytest.approx(25e-5, rel=1e-12)
    ids = b.gpu.handle.ids()            # order after the resume's sort, in snapshot (= a's) order
    b.Step(substeps=25)
    out_b = b.gpu.hssoa
    assert out_b.shape == out_a.shape
    ref = out_a[:, ids]
    tol = 1e-10 if precision == PRECISION_FP64 else 1e-6
    assert np.abs(out_b[POSX:POSX + 3] - ref[POSX:POSX + 3]).max() < tol
    assert np.abs(b.gpu.indenter_force - a.gpu.indenter_force).max() <= 1e-3 * np.abs(a.gpu.indenter_force).max()


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED])
def test_water_tank_setup_through_the_gpu_step(tmp_path, precision):
    """SetupType 2 (input_data/tank1b.json's setup): the points outside the
    centred BlockCutout become liquid at load (MarkSolidAndLiquid), the grid
    update drops the indenter, the floor only stops downward motion and
    DragGlobal damps every node (mpm_kernels.cuh:173-226); liquid points
    carry LiquidParticleMass and the water pressure. The water model takes
    the ice's kappa with gamma = 3, so the parameters follow tank1b.json's
    regime (E = 1e8, ice density 200) to keep the water's CFL number < 0.5."""
    js = write_case(tmp_path, SetupType=2, BlockCutout=[0.2, 0.1, 0.1], YoungsModulus=1e8, Density=200)
    model = Model3D.from_config(js, base_dir=tmp_path, precision=precision)
    p = model.prms
    p.DragGlobal = 2e-3
    model.Prepare()
    held = model.gpu.hssoa
    liquid = (held[0].view(np.int64) & STATUS_LIQUID) != 0
    n = held.shape[1]
    assert 0.3 * n < liquid.sum() < 0.9 * n
    q, soa, cap = snapshot.load_raw_points(str(tmp_path / "pc.h5"), parsed(js))
    perm = po.sort_permutation(q, soa, n)
    ref0 = np.ascontiguousarray(soa[:, perm])
    assert np.array_equal(held[0], ref0[0])        # same status words, liquid bits included
    steps = 100
    hist = model.gpu.handle.step(steps)
    assert np.all(hist == 0)                        # no indenter in this setup
    sim = po.OracleSim(p, ref0, n, svd_mode=0 if precision == PRECISION_FP64 else 1)
    _, err = sim.step(steps)
    assert err == 0
    out = model.gpu.handle.download()
    dv = np.abs(out[VELX:VELX + 3] - sim.soa[VELX:VELX + 3]).max() / np.abs(sim.soa[VELX:VELX + 3]).max()
    dx = np.abs(out[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max()
    assert np.abs(sim.soa[VELX + 1]).max() > 1e-3     # gravity has moved the water
    if precision == PRECISION_FP64:
        assert dx < 1e-12 and dv < 1e-9, (dx, dv)
    else:
        assert dx < 1e-6 and dv < 1e-3, (dx, dv)
