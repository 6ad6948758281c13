"""SimParams3D defaults, JSON reader and derived constants against the
formulas of parameters_sim_3d.cpp (Reset :5-62, ComputeHelperVariables
:65-86, ParseFile :89-162, ComputeLame/ComputeCamClayParams :164-175)."""
import ctypes
import glob
import math
import os

import pytest

from icempm_3dm_b200._lib import LIB, SimParams3D

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_text(text):
    p = SimParams3D()
    raw = ctypes.create_string_buffer(256)
    rc = LIB.mpm_params_parse_string(p, text.encode(), raw, 256)
    return rc, p, raw.value.decode()


def derived_ok(p):
    E, nu = p.YoungsModulus, p.PoissonsRatio
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    assert p.lambda_ == pytest.approx(lam, rel=1e-15)
    assert p.mu == pytest.approx(mu, rel=1e-15)
    assert p.kappa == pytest.approx(mu * 2. / 3. + lam, rel=1e-15)
    assert p.NACC_beta == pytest.approx(p.IceTensileStrength / p.IceCompressiveStrength, rel=1e-15)
    h = p.DomainDimensionX / p.GridXTotal
    assert p.cellsize == pytest.approx(h, rel=1e-15)
    assert p.cellsize_inv == pytest.approx(1 / h, rel=1e-15)
    assert p.Dp_inv == pytest.approx(4 / h ** 2, rel=1e-15)
    assert p.UpdateEveryNthStep == int(1.0 / (200 * p.InitialTimeStep))
    assert p.IndRSq == pytest.approx(p.IndDiameter ** 2 / 4, rel=1e-15)
    assert p.dt_vol_Dpinv == pytest.approx(p.InitialTimeStep * p.ParticleVolume * 4 / h ** 2, rel=1e-15)
    assert p.dt_Gravity == pytest.approx(p.InitialTimeStep * p.Gravity, rel=1e-15)
    assert p.vmax == pytest.approx(0.5 * h / p.InitialTimeStep, rel=1e-15)
    assert p.gbOffset == p.GridZ * p.GridY * p.GridHaloSize
    assert p.IndenterSubdivisions == int(math.pi * p.IndDiameter / h)


def test_reset_defaults():
    p = SimParams3D()
    LIB.mpm_params_reset(p)
    assert p.InitialTimeStep == 3e-5 and p.YoungsModulus == 5e8
    assert (p.GridXTotal, p.GridY, p.GridZ) == (128, 55, 55)
    assert p.DomainDimensionX == 3.33 and p.Density == 916 and p.PoissonsRatio == 0.3
    assert p.IndDiameter == 0.324 and p.IndVelocity == 0.2 and p.IndDepth == 0.25
    assert p.IceCompressiveStrength == 100e6 and p.IceTensileStrength == 10e6
    assert p.IceShearStrength == 6e6 and p.IceTensileStrength2 == 5e6
    assert p.DP_tan_phi == pytest.approx(math.tan(math.radians(45)), rel=1e-15)
    assert p.DP_threshold_p == 1e2 and p.GrainVariability == 0.5
    assert (p.tpb_P2G, p.tpb_Upd, p.tpb_G2P) == (256, 512, 128)
    assert p.GridHaloSize == 15 and p.nPartitions == 4 and p.SnapshotPeriod == 100
    derived_ok(p)


def test_parse_fixture():
    with open(os.path.join(HERE, "golden", "config_indentation.json")) as f:
        rc, p, raw = parse_text(f.read())
    assert rc == 0 and raw == "geometries_3d/3d_200k.h5"
    assert p.GridXTotal == 120 and p.GridY == 58 and p.DomainDimensionX == 1.2
    assert p.DP_tan_phi == pytest.approx(math.tan(math.radians(62)), rel=1e-15)
    assert list(p.BlockCutout) == [0.5, 0.25, 0.25]
    assert (p.tpb_P2G, p.tpb_Upd, p.tpb_G2P) == (128, 256, 64)
    assert p.animation_threshold_pos == 2e-3
    derived_ok(p)


def test_parse_file_and_errors(tmp_path):
    p = SimParams3D()
    raw = ctypes.create_string_buffer(64)
    assert LIB.mpm_params_parse_file(p, str(tmp_path / "missing.json").encode(), raw, 64) == 104
    bad = tmp_path / "bad.json"
    bad.write_text("{ not json")
    assert LIB.mpm_params_parse_file(p, str(bad).encode(), raw, 64) == 105
    nokey = tmp_path / "nokey.json"
    nokey.write_text('{"GridX": 10}')
    assert LIB.mpm_params_parse_file(p, str(nokey).encode(), raw, 64) == 106
    wrongtype = tmp_path / "wrong.json"
    wrongtype.write_text('{"InputRawPoints": "a.h5", "GridX": 10.5}')
    assert LIB.mpm_params_parse_file(p, str(wrongtype).encode(), raw, 64) == 105
    ok = tmp_path / "ok.json"
    ok.write_text('{"InputRawPoints": "pts.h5", "GridX": 200, "DP_phi": 30}')
    assert LIB.mpm_params_parse_file(p, str(ok).encode(), raw, 64) == 0
    assert raw.value == b"pts.h5" and p.GridXTotal == 200


def test_reference_input_files_parse_when_present():
    from oracle import pyoracle as po
    ref = po.reference_tree()
    files = sorted(glob.glob(os.path.join(ref, "input_data", "*.json"))) if ref else []
    if not files:
        pytest.skip("reference tree not present")
    for path in files:
        p = SimParams3D()
        raw = ctypes.create_string_buffer(256)
        assert LIB.mpm_params_parse_file(p, path.encode(), raw, 256) == 0, path
        assert raw.value
        derived_ok(p)
