"""Seeded synthetic block generator: counter-based RNG, lattice, placement
as SnapshotManager::LoadRawPoints (snapshotmanager.cpp:57-99)."""
import math

import numpy as np

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import FE00, IDX_JP_INV, POSX


def test_splitmix64_published_first_output():
    # first output of the splitmix64 generator started from state 0
    assert int(gen.splitmix64(np.uint64(0))) == 0xE220A8397B1DCDAF


def test_uniform_and_normal_are_deterministic():
    idx = np.arange(10000, dtype=np.uint64)
    a = gen.uniform(4, idx, 1)
    assert np.array_equal(a, gen.uniform(4, idx, 1))
    assert not np.array_equal(a, gen.uniform(5, idx, 1))
    assert 0 <= a.min() and a.max() < 1 and abs(a.mean() - 0.5) < 0.01
    z = gen.normal(4, idx, 3)
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.03


def test_lattice_counts_and_extent():
    pos = gen.jittered_lattice(50000, (1.0, 0.5, 0.5), seed=0)
    assert pos.shape == (3, 50000)
    assert pos.min() >= 0 and np.all(pos.max(axis=1) <= np.array([1.0, 0.5, 0.5]))
    pos2 = gen.jittered_lattice(50000, (1.0, 0.5, 0.5), seed=0)
    assert np.array_equal(pos, pos2)


def test_block_placement_and_initial_state():
    prms, soa, coh = gen.make_block(gen.CONFIGS["calib500k"], n=20000)
    h = prms.cellsize
    assert soa[POSX + 1].min() == 2 * h
    assert coh is None
    assert np.all(soa[IDX_JP_INV] == 1.0)
    assert np.all(soa[FE00] == 1.0) and np.all(soa[FE00 + 1] == 0.0)
    r = prms.IndDiameter / 2
    x_off = (prms.GridXTotal * h - (prms.xmax - prms.xmin)) / 2
    assert prms.indenter_x == math.floor((x_off - r) / h) * h
    assert prms.indenter_y == prms.ymax + 2 * h - prms.ymin + (r - prms.IndDepth)
    assert prms.ParticleVolume == prms.Volume / 20000 * 1.0 or prms.ParticleVolume > 0


def test_lognormal_cohesion():
    cfg = gen.CONFIGS["block2m"]
    _, _, coh = gen.make_block(cfg, n=100000)
    assert coh is not None and coh.shape == (100000,)
    lg = np.log(coh / 3e5)
    assert abs(np.median(lg)) < 0.01 and abs(lg.std() - 0.3) < 0.01
