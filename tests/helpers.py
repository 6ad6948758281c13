"""Shared inputs for the parity tests: seeded small blocks and perturbed
particle states that exercise the elastic, crushed, tension and liquid
branches of the step."""
import numpy as np

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200.layout import (BP00, FE00, IDX_JP_INV, IDX_UTILITY, STATUS_CRUSHED,
                                  STATUS_LIQUID, VELX)


def util_as_double(bits):
    return np.asarray(bits, dtype=np.int64).view(np.float64)


def util_bits(soa):
    return soa[IDX_UTILITY].view(np.int64)


def perturbed_block(n=3000, seed=11, crushed_frac=0.15, strong_frac=0.1, tension_frac=0.03, liquid_frac=0.0,
                    dims=(0.2, 0.1, 0.1), h=0.01, ind_velocity=0.2, youngs=5e8, ops=None):
    """A small block whose particles carry velocity, affine velocity and
    elastic strain; some are pre-crushed, some strongly strained, a few in
    tension with Jp_inv < 1. ops: the SimParams3D routines of the generator
    (default: the library's)."""
    prms, soa, _ = gen.small_block(n=n, seed=seed, dims=dims, h=h, ind_velocity=ind_velocity, youngs=youngs,
                                   ops=ops)
    n = soa.shape[1]
    rng = np.random.default_rng(seed)
    soa[VELX:VELX + 3] = 0.05 * rng.standard_normal((3, n))
    soa[BP00:BP00 + 9] = 5.0 * rng.standard_normal((9, n))
    E = 2e-4 * rng.standard_normal((9, n))
    strong = rng.random(n) < strong_frac
    E[:, strong] *= 150.0
    soa[FE00:FE00 + 9] += E
    bits = np.zeros(n, dtype=np.int64)
    crushed = rng.random(n) < crushed_frac
    bits[crushed] |= STATUS_CRUSHED
    tension = rng.random(n) < tension_frac
    bits[tension] |= STATUS_CRUSHED
    soa[IDX_JP_INV, tension] = 0.995
    if liquid_frac > 0:
        liquid = rng.random(n) < liquid_frac
        bits[liquid] |= STATUS_LIQUID
    soa[IDX_UTILITY] = util_as_double(bits)
    return prms, soa


def close(a, b, rtol, atol_scale=1e-12):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.allclose(a, b, rtol=rtol, atol=atol_scale * scale), float(np.max(np.abs(a - b)) / scale)
