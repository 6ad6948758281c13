"""GPU parity of the mixed-precision step (FP32 state and transfers, FP64
SVD / return map / force reduction) against the FP64 oracle with the FP64
SVD variant, through the C-ABI.

Tolerances (FP32 arithmetic): per-field single-step relative deviation
<= 2e-5 of the field's magnitude, positions <= 1e-7 m absolute; the
indenter force history over 60 substeps within 1e-3 relative (the north
star's bound for the mixed form).
"""
import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_MIXED
from icempm_3dm_b200._lib import BP00, FE00, IDX_JP_INV, IDX_UTILITY, POSX, STATUS_CRUSHED, VELX
from oracle import pyoracle as po
from tests.helpers import perturbed_block, util_bits

pytestmark = pytest.mark.gpu


def rel_dev(a, b):
    return float(np.max(np.abs(a - b)) / max(np.abs(b).max(), 1e-300))


def test_upload_download_round_trip():
    prms, soa = perturbed_block(n=3000, seed=71)
    with MPMHandle(prms, soa.shape[1], PRECISION_MIXED) as h:
        h.upload(soa)
        out = h.download()
    assert np.abs(out[POSX:POSX + 3] - soa[POSX:POSX + 3]).max() < 2e-8
    assert rel_dev(out[VELX:VELX + 3], soa[VELX:VELX + 3]) < 1e-7
    assert np.abs(out[FE00:FE00 + 9] - soa[FE00:FE00 + 9]).max() < 1e-8
    assert rel_dev(out[BP00:BP00 + 9], soa[BP00:BP00 + 9]) < 1e-7
    assert np.array_equal(util_bits(out), util_bits(soa))


def test_single_step_phases_close_to_oracle():
    prms, soa = perturbed_block(n=4000, seed=31)
    n = soa.shape[1]
    ix = prms.indenter_x + 0.02
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.upload(soa)
        h.reset_indenter_force_accumulator()
        h.reset_grid()
        h.p2g()
        acc = h.grid(0)
        h.update_nodes(ix, prms.indenter_y)
        vel = h.grid(1)
        h.g2p(True)
        out = h.download()
    ref_grid, _ = po.p2g(prms, soa, n)
    assert rel_dev(acc[0], ref_grid[0]) < 1e-6
    for c in range(1, 4):
        assert rel_dev(acc[c], ref_grid[c]) < 2e-5, c
    mass = ref_grid[0].copy()
    po.update_nodes(prms, ref_grid, ix, prms.indenter_y)
    live = mass > 1e-3 * mass.max()
    for c in range(1, 4):
        assert rel_dev(vel[c][live], ref_grid[c][live]) < 2e-5, c
    ref = soa.copy()
    po.g2p(prms, ref, n, ref_grid, record_pq=True, svd_mode=1)
    crushed_ref = (util_bits(ref) & STATUS_CRUSHED) != 0
    crushed = (util_bits(out) & STATUS_CRUSHED) != 0
    assert np.mean(crushed != crushed_ref) < 1e-3
    same = crushed == crushed_ref
    assert np.abs(out[POSX:POSX + 3] - ref[POSX:POSX + 3]).max() < 1e-7
    assert rel_dev(out[VELX:VELX + 3], ref[VELX:VELX + 3]) < 2e-5
    assert rel_dev(out[BP00:BP00 + 9], ref[BP00:BP00 + 9]) < 2e-5
    dF = np.abs(out[FE00:FE00 + 9][:, same] - ref[FE00:FE00 + 9][:, same]).max()
    assert dF < 2e-6, dF
    assert rel_dev(out[IDX_JP_INV][same], ref[IDX_JP_INV][same]) < 1e-5


def test_force_history_within_1e3_of_fp64():
    prms, soa = perturbed_block(n=3000, seed=41, ind_velocity=0.5, crushed_frac=0.05, strong_frac=0.0)
    n = soa.shape[1]
    steps = 60
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.upload(soa)
        hist = h.step(steps)
        out = h.download()
    sim = po.OracleSim(prms, soa, n, svd_mode=1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    norm = np.linalg.norm(ref_hist)
    assert norm > 0
    assert np.linalg.norm(hist - ref_hist) / norm < 1e-3
    assert np.abs(out[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < 1e-6


def test_sort_in_mixed_mode_matches_oracle_permutation():
    prms, soa = perturbed_block(n=4000, seed=81)
    n = soa.shape[1]
    rng = np.random.default_rng(2)
    soa = np.ascontiguousarray(soa[:, rng.permutation(n)])
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.upload(soa)
        held = h.download()          # positions as the mixed state holds them
        h.sort()
        ids = h.ids()
        out = h.download()
    perm = po.sort_permutation(prms, held, n)
    assert np.array_equal(ids, perm)
    assert np.array_equal(out, held[:, perm])


def test_split_calls_and_periodic_sort_keep_state():
    """The fused kernel writes v and C only on the last substep of a call and
    before a sort; a run split over calls with sorts in between must carry the
    same state as one call and stay on the FP64 oracle."""
    prms, soa = perturbed_block(n=3000, seed=43, ind_velocity=0.5, crushed_frac=0.05, strong_frac=0.0)
    n = soa.shape[1]
    steps = 30
    outs = []
    for chunks in ((30,), (10, 7, 13)):
        with MPMHandle(prms, n, PRECISION_MIXED) as h:
            h.upload(soa)
            h.set_sort_interval(4)
            hist = np.concatenate([h.step(c) for c in chunks])
            out = h.download()
            ids = h.ids()
        full = np.zeros_like(out)
        full[:, ids] = out
        outs.append((hist, full))
    sim = po.OracleSim(prms, soa, n, svd_mode=1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    for hist, full in outs:
        assert np.linalg.norm(hist - ref_hist) / np.linalg.norm(ref_hist) < 1e-3
        assert np.abs(full[POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < 1e-6
        assert rel_dev(full[VELX:VELX + 3], sim.soa[VELX:VELX + 3]) < 1e-3
        assert rel_dev(full[BP00:BP00 + 9], sim.soa[BP00:BP00 + 9]) < 1e-3
    (h1, f1), (h2, f2) = outs
    assert np.abs(f1[VELX:VELX + 3] - f2[VELX:VELX + 3]).max() < 1e-4 * np.abs(f1[VELX:VELX + 3]).max()


def test_liquid_and_disabled_particles_in_the_fused_path():
    """Water points (status 0x40000: Kirchhoff stress replaced by the water
    pressure, Jp_inv advected by det(I + dt C)) and disabled points (skipped)
    through the mixed fused kernel, against the FP64-SVD oracle."""
    from icempm_3dm_b200._lib import STATUS_DISABLED
    from tests.helpers import util_as_double
    prms, soa = perturbed_block(n=4000, seed=91, liquid_frac=0.15, crushed_frac=0.05, strong_frac=0.0,
                                ind_velocity=0.5)
    n = soa.shape[1]
    bits = util_bits(soa).copy()
    # water starts unstrained (Jp_inv = 1): a block's "tension" points made
    # liquid would start as water under -6 MPa, a state whose dynamics amplify
    # any rounding difference (mixed and FP64 then part within 20 substeps)
    # and without the block's random affine field (std 5 1/s), which compresses the
    # water by tens of per cent within 30 substeps
    soa[IDX_JP_INV, (bits & (1 << 18)) != 0] = 1.0
    soa[BP00:BP00 + 9, (bits & (1 << 18)) != 0] = 0.0
    dis = np.random.default_rng(3).random(n) < 0.05
    bits[dis] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    steps = 30
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.upload(soa)
        held = h.download()         # the state as the mixed handle holds it (FP32 rounding)
        hist = h.step(steps)
        out = h.download()
    sim = po.OracleSim(prms, soa, n, svd_mode=1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    assert np.linalg.norm(hist - ref_hist) / np.linalg.norm(ref_hist) < 1e-3
    live = ~dis
    assert np.array_equal(out[:, dis], held[:, dis])              # disabled points untouched
    # positions: FP32 state in a block with holes and a random affine field
    # (std 5 1/s) on its solid points; 1.2e-6 m measured after 30 substeps
    xdev = np.abs(out[POSX:POSX + 3, live] - sim.soa[POSX:POSX + 3, live]).max()
    assert xdev < 5e-6, xdev
    liquid = (bits & (1 << 18)) != 0
    # water Jp_inv: compared where no return map can touch it (not crushed)
    crushed_any = ((util_bits(out) | util_bits(sim.soa)) & STATUS_CRUSHED) != 0
    wl = live & liquid & ~crushed_any
    assert wl.sum() > 100
    # the reference's water uses the ice bulk modulus (kappa ~ 4e8 Pa): its points
    # reach J = 0.87..1.45 here, and Jp_inv follows the oracle to 2e-3 of that
    assert rel_dev(out[IDX_JP_INV, wl], sim.soa[IDX_JP_INV, wl]) < 2e-3


def test_fixed_point_accumulation_is_exact_and_repeatable():
    """MPM_ACCUM_FIXED: the mixed P2G sums in 64-bit fixed point. The grid
    after P2G matches the oracle as the float4 sums do (2e-5), the force
    history stays within 1e-3 of the FP64 oracle, and two runs of the same
    input give bit-identical particle states (the float4 atomics' sums depend
    on the order of the adds; the integer sums do not)."""
    from icempm_3dm_b200.layout import ACCUM_FIXED
    prms, soa = perturbed_block(n=3000, seed=41, ind_velocity=0.5, crushed_frac=0.05, strong_frac=0.0)
    n = soa.shape[1]
    with MPMHandle(prms, n, PRECISION_MIXED) as h:
        h.set_grid_accumulation(ACCUM_FIXED)
        h.upload(soa)
        h.reset_grid()
        h.p2g()
        acc = h.grid(0)
    ref_grid, _ = po.p2g(prms, soa, n)
    assert rel_dev(acc[0], ref_grid[0]) < 1e-6
    for c in range(1, 4):
        assert rel_dev(acc[c], ref_grid[c]) < 2e-5, c
    steps = 60
    runs = []
    for _ in range(2):
        with MPMHandle(prms, n, PRECISION_MIXED) as h:
            h.set_grid_accumulation(ACCUM_FIXED)
            h.upload(soa)
            hist = h.step(steps)
            runs.append((hist, h.download()))
    sim = po.OracleSim(prms, soa, n, svd_mode=1)
    ref_hist, err = sim.step(steps)
    assert err == 0
    assert np.linalg.norm(runs[0][0] - ref_hist) / np.linalg.norm(ref_hist) < 1e-3
    assert np.abs(runs[0][1][POSX:POSX + 3] - sim.soa[POSX:POSX + 3]).max() < 1e-6
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.allclose(runs[0][0], runs[1][0], rtol=1e-12, atol=0)
