"""bench.py's reference arm on CPU: the reference's own step kernels (host
build, oracle/_ref) or, without that build, the oracle port run exactly
--steps substeps, each over a bounded sample of the workload, and print the
contract's JSON line; the product library is never loaded by that arm."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from icempm_3dm_b200 import generator as gen  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

KIND = "reference" if po.ref_mpm_lib() is not None else "port"


def run_arm(*extra):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *extra],
                       capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("ref_seconds,sampled", [(60.0, False), (0.02, True)])
def test_reference_arm_times_exactly_k_steps(ref_seconds, sampled):
    d = run_arm("--workload", "block250k", "--steps", "4", "--warmup", "1", "--ref-seconds", str(ref_seconds))
    assert d["impl"] == "reference" and d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["steps"] == 4 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"] == {"workload": "block250k", "particles": 250_000}
    base = d["cpu_baseline"]
    assert base["value"] == d["value"] and base["kind"] == KIND and base["cores"] >= 1
    assert base["sample"].startswith("4 substeps of ")
    assert ("block of the block250k workload" in base["sample"]) == sampled
    assert d["e2e"] == {"value": d["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("name", ["block8m", "grains30m"])
def test_reference_sample_keeps_density_and_scales_the_grid(name):
    cfg = gen.CONFIGS[name]
    s = bench.reference_sample(cfg, cfg.n // 10)
    assert s.n == cfg.n // 10
    vol = lambda c: c.dims[0] * c.dims[1] * c.dims[2]
    assert abs(s.n / vol(s) - cfg.n / vol(cfg)) < 1e-9 * cfg.n / vol(cfg)
    assert (s.h, s.dt, s.seed, s.ind_velocity, s.cohesion_sigma_log) == \
        (cfg.h, cfg.dt, cfg.seed, cfg.ind_velocity, cfg.cohesion_sigma_log)
    if cfg.grains:
        assert s.grains == round(cfg.grains / 10)
    gs, gf = gen.grid_dims(s), gen.grid_dims(cfg)
    assert gs[0] < gf[0] and gs[1:] == gf[1:]   # the grid shrinks in x only


def test_reference_arm_does_not_load_the_product_library():
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'block250k', '--steps', '2', "
            "'--warmup', '1', '--ref-seconds', '0.02']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_LIB_LOADED' if 'libicempm_b200' in maps else 'PRODUCT_LIB_ABSENT'); "
            "print('REF_LIB_LOADED' if 'libref_mpm' in maps else 'REF_LIB_ABSENT')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_LIB_ABSENT" in r.stdout
    if KIND == "reference":
        assert "REF_LIB_LOADED" in r.stdout
