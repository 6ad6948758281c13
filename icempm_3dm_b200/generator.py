"""Seeded synthetic ice blocks for the indentation setup.

The reference reads gmsh/Poisson-disk point clouds from HDF5
(SnapshotManager::LoadRawPoints, snapshotmanager.cpp:20-113). This module
generates a stand-in with the shapes and sizes of the benchmark workloads:
a jittered cubic lattice, seeded by a counter-based RNG (splitmix64, keyed by
seed, particle index and stream), then placed and initialised exactly as
LoadRawPoints does:
  - block offset: x centred in the domain, lowest point at y = 2h, z centred
    (snapshotmanager.cpp:57-75);
  - F = I, Jp_inv = 1 (HostSideSOA::InitializeBlock, host_side_soa.cpp:88-97);
  - indenter start x = floor((block_left - sqrt(r^2 - (r-IndDepth)^2))/h) h,
    y = block_top + r - IndDepth (snapshotmanager.cpp:82-96);
  - ParticleVolume = Volume / N (:99).
Per-particle cohesion (lognormal) is drawn from the same RNG.

The parameter block's defaults and derived constants come from a set of
SimParams3D routines, `ops` (Reset, SetPhi, ComputeCamClayParams,
ComputeHelperVariables): by default the library's own (mpm_params_*); any
other set with the same meaning can be passed. This module loads the library
only when the default set is used.
"""
import dataclasses
import math
from collections import namedtuple

import numpy as np

from .layout import FE00, IDX_JP_INV, N_PTS_ARRAYS, POSX, SimParams3D

ParamOps = namedtuple("ParamOps", "reset set_phi compute_camclay compute_helper_variables")


def library_param_ops():
    """The library's SimParams3D routines (include/icempm_b200.h)."""
    from ._lib import LIB
    return ParamOps(LIB.mpm_params_reset, LIB.mpm_params_set_phi, LIB.mpm_params_compute_camclay,
                    LIB.mpm_params_compute_helper_variables)

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    """splitmix64 finaliser (Steele, Lea, Flood 2014), vectorised on uint64."""
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(seed, idx, stream):
    """Uniform doubles in [0, 1) for particle indices idx (counter-based)."""
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed) * np.uint64(0x632BE59BD9B4E019) + np.uint64(stream))
        r = splitmix64(key ^ (idx * np.uint64(0xD1B54A32D192ED03)))
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed, idx, stream):
    """Standard normal deviates by Box-Muller on two uniform streams."""
    u1 = uniform(seed, idx, 2 * stream + 1000)
    u2 = uniform(seed, idx, 2 * stream + 1001)
    u1 = np.maximum(u1, 1e-300)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def jittered_lattice(n, dims, seed, jitter=0.3):
    """n points in the box [0, dims] on a jittered cubic lattice.

    Spacing s = (V/n)^(1/3); per-axis counts ceil(L/s) (spacing adjusted to
    fill the box); if the lattice holds more than n sites, a seeded subset of
    n sites is kept in lattice order (x slowest, z fastest). Each coordinate
    moves by a uniform +-jitter * spacing.
    """
    L = np.asarray(dims, dtype=np.float64)
    s = (L.prod() / n) ** (1.0 / 3.0)
    counts = np.maximum(1, np.ceil(L / s - 1e-9).astype(np.int64))
    total = int(counts.prod())
    if total < n:
        raise ValueError("lattice smaller than n")
    sites = np.arange(total, dtype=np.int64)
    if total > n:
        u = uniform(seed, sites, 7)
        keep = np.argpartition(u, n)[:n]
        sites = np.sort(keep)
    nz, ny = counts[2], counts[1]
    ix = sites // (ny * nz)
    iy = (sites // nz) % ny
    iz = sites % nz
    sp = L / counts
    pid = np.arange(n, dtype=np.uint64)
    pos = np.empty((3, n))
    for d, ii in enumerate((ix, iy, iz)):
        j = (2.0 * uniform(seed, pid, d) - 1.0) * jitter
        pos[d] = (ii + 0.5 + j) * sp[d]
    return pos


@dataclasses.dataclass
class BlockConfig:
    """One indentation workload (block on a sticky floor, cylinder moving +x)."""
    name: str
    n: int
    dims: tuple
    h: float
    seed: int
    dt: float
    steps: int
    ind_velocity: float
    cohesion_median: float = 3.0e5
    cohesion_sigma_log: float = 0.0          # 0: uniform cohesion
    density: float = 917.0
    youngs: float = 5.0e8
    poisson: float = 0.3
    phi_deg: float = 62.0
    ind_radius: float = 0.05
    pad: int = 3                              # wall pad nodes per side
    halo: int = 0                             # GridHaloSize (one partition)
    grains: int = 0                           # spherical grains above a lattice block (0: plain block)
    grain_frac: float = 0.0                   # share of the particles in the grains
    grain_r: tuple = (0.02, 0.06)             # grain radius range (uniform)
    block_frac_y: float = 0.4                 # lattice block height / domain height (grains cases)


CONFIGS = {
    "block250k": BlockConfig("block250k", 250_000, (1.0, 0.5, 0.5), 0.01, 0, 1e-5, 1000, 0.2),
    "block2m": BlockConfig("block2m", 2_000_000, (2.0, 1.0, 1.0), 0.0125, 1, 5e-6, 2000, 0.5,
                           cohesion_sigma_log=0.3),
    "block8m": BlockConfig("block8m", 8_000_000, (4.0, 1.0, 1.0), 0.01, 2, 5e-6, 2000, 1.0,
                           cohesion_sigma_log=0.3),
    "calib500k": BlockConfig("calib500k", 500_000, (1.0, 0.5, 0.5), 0.01, 3, 1e-5, 200, 0.2),
    # non-uniform density: 70 % in a lattice block filling the lower 40 % of a
    # 6.0 x 1.5 x 1.5 m domain, 30 % in 20,000 grains above it
    "grains30m": BlockConfig("grains30m", 30_000_000, (6.0, 1.5, 1.5), 0.008, 4, 2e-6, 5000, 2.0,
                             cohesion_sigma_log=0.5, grains=20_000, grain_frac=0.3),
}


def grid_dims(cfg):
    """Nodes: block cells + wall pads; in x also room for the indenter on the
    -x side (centred block, as LoadRawPoints centres it); in y the block
    stands 2h above the floor."""
    nb = [int(math.ceil(L / cfg.h - 1e-9)) for L in cfg.dims]
    clear = int(math.ceil(cfg.ind_radius / cfg.h)) + 2
    gx = nb[0] + 2 * (cfg.pad + clear)
    gy = nb[1] + 2 + cfg.pad + 3
    gz = nb[2] + 2 * cfg.pad + 2
    return gx, gy, gz


def make_params(cfg, n=None, ops=None):
    """SimParams3D for cfg; defaults and derived constants by ops.reset /
    ops.compute_camclay / ops.compute_helper_variables (default: the
    library's own)."""
    ops = ops or library_param_ops()
    p = SimParams3D()
    ops.reset(p)
    gx, gy, gz = grid_dims(cfg)
    p.GridXTotal, p.GridY, p.GridZ = gx, gy, gz
    p.DomainDimensionX = gx * cfg.h
    p.GridHaloSize = cfg.halo
    p.nPartitions = 1
    p.InitialTimeStep = cfg.dt
    p.YoungsModulus = cfg.youngs
    p.PoissonsRatio = cfg.poisson
    p.Density = cfg.density
    ops.set_phi(p, cfg.phi_deg)
    p.DP_threshold_p = cfg.cohesion_median / p.DP_tan_phi
    p.GrainVariability = 0.0
    p.IndDiameter = 2 * cfg.ind_radius
    p.IndVelocity = cfg.ind_velocity
    p.IndDepth = cfg.ind_radius
    p.nPtsTotal = cfg.n if n is None else n
    p.Volume = float(np.prod(cfg.dims))
    ops.compute_camclay(p)
    ops.compute_helper_variables(p)
    return p


def make_block(cfg, n=None, ops=None):
    """(prms, soa, cohesion): soa is a (28, n) float64 host SoA in the
    reference layout; cohesion is None for uniform cohesion. ops: the
    SimParams3D routines (default: the library's)."""
    ops = ops or library_param_ops()
    if cfg.grains > 0:
        return make_grains_block(cfg, n, ops)
    n = cfg.n if n is None else n
    dims = cfg.dims
    if n != cfg.n:   # a smaller copy of the same block keeps the spacing
        scale = (n / cfg.n) ** (1.0 / 3.0)
        dims = tuple(d * scale for d in cfg.dims)
        cfg = dataclasses.replace(cfg, dims=dims, n=n)
    p = make_params(cfg, n, ops)
    pos = jittered_lattice(n, dims, cfg.seed)
    h = p.cellsize
    mins, maxs = pos.min(axis=1), pos.max(axis=1)
    box_x, box_z = p.GridXTotal * h, p.GridZ * h
    x_off = (box_x - (maxs[0] - mins[0])) / 2
    y_off = 2 * h - mins[1]
    z_off = (box_z - (maxs[2] - mins[2])) / 2
    pos[0] += x_off
    pos[1] += y_off
    pos[2] += z_off
    p.xmin, p.ymin, p.zmin = mins
    p.xmax, p.ymax, p.zmax = maxs
    block_left = x_off
    block_top = p.ymax + y_off
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    x_ind_offset = math.sqrt(r * r - ht * ht)
    p.indenter_x = math.floor((block_left - x_ind_offset) / h) * h
    p.indenter_y = block_top + ht
    p.indenter_x_initial = p.indenter_x
    p.indenter_y_initial = p.indenter_y
    p.ParticleVolume = p.Volume / n
    ops.compute_helper_variables(p)

    soa = np.zeros((N_PTS_ARRAYS, n), dtype=np.float64)
    soa[POSX:POSX + 3] = pos
    soa[IDX_JP_INV] = 1.0
    for i in range(3):
        soa[FE00 + 4 * i] = 1.0
    cohesion = None
    if cfg.cohesion_sigma_log > 0:
        z = normal(cfg.seed, np.arange(n, dtype=np.uint64), 11)
        cohesion = cfg.cohesion_median * np.exp(cfg.cohesion_sigma_log * z)
    return p, soa, cohesion


def make_grains_block(cfg, n=None, ops=None):
    """The non-uniform stress case: (1 - grain_frac) of the particles on a
    jittered lattice filling the lower block_frac_y of the domain (placed as
    make_block places a block), grain_frac of them in cfg.grains spheres with
    radii uniform in cfg.grain_r whose centres are drawn uniformly (Poisson,
    overlaps allowed) in the domain above the block; each sphere holds a share
    of those particles proportional to its volume, spread uniformly inside it.
    Every particle has the lattice's particle volume. A smaller n scales the
    domain and the grain count with the particle count."""
    ops = ops or library_param_ops()
    n = cfg.n if n is None else n
    if n != cfg.n:
        scale = (n / cfg.n) ** (1.0 / 3.0)
        cfg = dataclasses.replace(cfg, dims=tuple(d * scale for d in cfg.dims), n=n,
                                  grains=max(1, int(round(cfg.grains * n / cfg.n))))
    n_grain = int(round(n * cfg.grain_frac))
    n_lat = n - n_grain
    dom = np.asarray(cfg.dims, dtype=np.float64)
    lat_dims = (dom[0], dom[1] * cfg.block_frac_y, dom[2])
    p = make_params(cfg, n, ops)
    h = p.cellsize
    lat = jittered_lattice(n_lat, lat_dims, cfg.seed)
    box_x, box_z = p.GridXTotal * h, p.GridZ * h
    x_off = (box_x - dom[0]) / 2
    y_off = 2 * h
    z_off = (box_z - dom[2]) / 2
    lat[0] += x_off
    lat[1] += y_off
    lat[2] += z_off
    # grains: radii, centres above the block, particle counts by volume
    g = np.arange(cfg.grains, dtype=np.uint64)
    r0, r1 = cfg.grain_r
    rad = r0 + (r1 - r0) * uniform(cfg.seed, g, 21)
    lat_top = y_off + lat_dims[1]
    cx = x_off + rad + (dom[0] - 2 * rad) * uniform(cfg.seed, g, 22)
    cy = lat_top + rad + (y_off + dom[1] - lat_top - 2 * rad) * uniform(cfg.seed, g, 23)
    cz = z_off + rad + (dom[2] - 2 * rad) * uniform(cfg.seed, g, 24)
    vol = rad ** 3
    counts = np.floor(n_grain * vol / vol.sum()).astype(np.int64)
    short = n_grain - int(counts.sum())
    counts[np.argsort(-(n_grain * vol / vol.sum() - counts))[:short]] += 1
    owner = np.repeat(np.arange(cfg.grains), counts)
    pid = np.arange(n_grain, dtype=np.uint64) + np.uint64(n_lat)
    d = np.stack([normal(cfg.seed, pid, 31 + k) for k in range(3)])
    d /= np.maximum(np.linalg.norm(d, axis=0), 1e-300)
    rr = rad[owner] * np.cbrt(uniform(cfg.seed, pid, 34))
    gpos = np.stack([cx[owner], cy[owner], cz[owner]]) + d * rr
    pos = np.concatenate([lat, gpos], axis=1)

    mins, maxs = pos.min(axis=1), pos.max(axis=1)
    p.xmin, p.ymin, p.zmin = mins
    p.xmax, p.ymax, p.zmax = maxs
    block_left = x_off
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    p.indenter_x = math.floor((block_left - math.sqrt(r * r - ht * ht)) / h) * h
    p.indenter_y = lat_top + ht
    p.indenter_x_initial = p.indenter_x
    p.indenter_y_initial = p.indenter_y
    p.Volume = float(np.prod(lat_dims)) * n / n_lat
    p.ParticleVolume = float(np.prod(lat_dims)) / n_lat
    ops.compute_helper_variables(p)

    soa = np.zeros((N_PTS_ARRAYS, n), dtype=np.float64)
    soa[POSX:POSX + 3] = pos
    soa[IDX_JP_INV] = 1.0
    for i in range(3):
        soa[FE00 + 4 * i] = 1.0
    z = normal(cfg.seed, np.arange(n, dtype=np.uint64), 11)
    cohesion = cfg.cohesion_median * np.exp(cfg.cohesion_sigma_log * z)
    return p, soa, cohesion


def small_block(n=4000, seed=5, dims=(0.2, 0.1, 0.1), h=0.01, dt=1e-5, ind_velocity=0.2,
                cohesion_sigma_log=0.0, youngs=5e8, halo=0, ops=None):
    """A small block for parity tests (seconds on the oracle)."""
    cfg = BlockConfig("small", n, dims, h, seed, dt, 0, ind_velocity, cohesion_sigma_log=cohesion_sigma_log,
                      youngs=youngs, halo=halo)
    return make_block(cfg, ops=ops)


def calibration_block(n=20_000, penetration_cells=3, ind_velocity=2.0, cohesion_sigma_log=0.3):
    """A smaller copy of the calib500k block (same spacing) for strength
    calibration, with the indenter started penetration_cells cells into the
    block and driven at ind_velocity: at calib500k's own 0.2 m/s over 200
    substeps the indenter travels 0.4 mm and no particle crushes, so the
    force history does not depend on cohesion at all."""
    cfg = dataclasses.replace(CONFIGS["calib500k"], ind_velocity=ind_velocity,
                              cohesion_sigma_log=cohesion_sigma_log)
    prms, soa, coh = make_block(cfg, n=n)
    prms.indenter_x_initial += penetration_cells * prms.cellsize
    prms.indenter_x = prms.indenter_x_initial
    return prms, soa, coh


__all__ = ["BlockConfig", "CONFIGS", "ParamOps", "library_param_ops", "make_block", "make_grains_block",
           "make_params", "small_block", "calibration_block",
           "jittered_lattice", "splitmix64", "uniform", "normal"]
