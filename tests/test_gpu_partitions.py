"""x-slab partitions on the GPU against the one-partition run.

The reference runs its partitions on however many devices there are
(GPU_Implementation6::initialize, gpu_implementation6.cpp:331-335); here 2 to
5 partitions share GPU 0. The block translates at 15 m/s in +x, so particles
cross the slab boundaries and move to the next partition; transfers run every
10 substeps. The block is lifted off the sticky floor and kept out of the
indenter's reach in the long runs: shearing or pushing it would start crush
and contact switches, after which two runs that differ only in the order of
the FP64 atomics part as far as any two do.

Checks against one partition on the same input (particles matched by id,
the partition bits of the status word masked):
  FP64: force history within 1e-9, state within 1e-9 of each field's
        largest magnitude (C 1e-8), status words equal;
  mixed: force history within 1e-4 (FP32 sums in another order), positions
        within 1e-6 m;
and that points did move (disabled counts), that a forced rebalance keeps
the run on the one-partition result, and that the indenter force of a node
in the overlap of two partitions is counted once (a boundary in the contact
zone with 5 partitions, 60 substeps in contact). The same run with one partition per process
(RankPartition, 2 processes on GPU 0 exchanging through gloo and host
memory) matches too.
"""
import os
import socket

import numpy as np
import pytest

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_MIXED
from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200.layout import IDX_UTILITY, POSX, VELX
from icempm_3dm_b200.partitions import PartitionedSim, sort_order
from tests.helpers import util_bits

pytestmark = pytest.mark.gpu

STEPS = 300
FIELDS = (("Jp_inv", 3, 4), ("x", 4, 7), ("v", 7, 10), ("F", 10, 19), ("C", 19, 28))


def moving_block(nparts, seed=71, contact=False):
    """The small block lifted 2 cells off the sticky floor (which would shear
    its bottom layer) and translating at 15 m/s in +x with a little noise in
    v and F. contact: the indenter 1 cell into the -x face, following at
    15.2 m/s; else it is out of reach and the force history is zero."""
    prms, soa, _ = gen.small_block(n=8000, seed=seed, dims=(0.2, 0.1, 0.1), halo=6)
    n = soa.shape[1]
    rng = np.random.default_rng(seed)
    soa[POSX + 1] += 2 * prms.cellsize
    soa[VELX] = 15.0
    soa[VELX:VELX + 3] += 0.01 * rng.standard_normal((3, n))
    soa[10:19] += 1e-5 * rng.standard_normal((9, n))
    prms.IndVelocity = 15.2
    if contact:
        prms.indenter_x_initial += 1 * prms.cellsize
        prms.indenter_y += 2 * prms.cellsize
    else:
        prms.indenter_x_initial = -10.0
    prms.indenter_x = prms.indenter_x_initial
    prms.indenter_y_initial = prms.indenter_y
    prms.UpdateEveryNthStep = 20
    prms.PointTransferFrequency = 2
    prms.nPartitions = nparts
    prms.VectorCapacity_transfer = 4000
    prms.RebalanceThresholdFreeSpaceRemaining = 0.0
    prms.RebalanceThresholdDisabledPercentage = 1.0
    return prms, soa


def one_partition(prms, soa, precision, steps=STEPS):
    n = soa.shape[1]
    order = sort_order(prms, soa, n)
    with MPMHandle(prms, n, precision) as h:
        h.upload(np.ascontiguousarray(soa[:, order]))
        h.upload_ids(order.astype(np.uint32))
        hist = h.step(steps)
        out, ids = h.download(), h.ids()
    full = np.zeros_like(out)
    full[:, ids] = out
    return hist, full


def by_id(out, ids, n):
    live = (util_bits(out) & 0x20000) == 0
    full = np.zeros((out.shape[0], n))
    full[:, ids[live]] = out[:, live]
    assert np.array_equal(np.sort(ids[live]), np.arange(n))     # every particle exactly once
    return full


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def compare(name, hist, full, ref_hist, ref_full, fp64):
    norm = np.linalg.norm(ref_hist)
    e = float(np.linalg.norm(hist - ref_hist) / norm) if norm > 0 else float(np.abs(hist).max())
    mask = np.int64(~(0xff << 24))
    stat_eq = np.array_equal(util_bits(full) & mask, util_bits(ref_full) & mask)
    errs = {f: rel(full[a:b], ref_full[a:b]) for f, a, b in FIELDS}
    print(f"\n{name}: force {e:.2e}, " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()) + f", status equal {stat_eq}")
    if fp64:
        assert e < 1e-9
        assert stat_eq
        for k, v in errs.items():
            # C is a difference quotient over h of node velocities near 15 m/s:
            # its rounding is 1/h times theirs, against a field of ~1 1/s
            assert v < (1e-8 if k == "C" else 1e-9), k
    else:
        assert e < 1e-4
        assert np.abs(full[POSX:POSX + 3] - ref_full[POSX:POSX + 3]).max() < 1e-6


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitions_match_one_partition(nparts, precision):
    prms, soa = moving_block(nparts)
    n = soa.shape[1]
    ref_hist, ref_full = one_partition(prms, soa, precision)
    with PartitionedSim(prms, n, precision) as m:
        m.upload(soa)
        info0 = m.info()
        hist = m.step(STEPS)
        info = m.info()
        out, ids = m.download()
    assert all(x0 + gxp == info0[i + 1][0] for i, (x0, gxp, _, _) in enumerate(info0[:-1]))
    moved = sum(nd for _, _, _, nd in info)
    assert moved > 0, info
    compare(f"{nparts} partitions ({'fp64' if precision == PRECISION_FP64 else 'mixed'}), {moved} moved",
            hist, by_id(out, ids, n), ref_hist, ref_full, precision == PRECISION_FP64)


def test_rebalance_keeps_the_run():
    prms, soa = moving_block(3, seed=72)
    prms.RebalanceThresholdDisabledPercentage = 1e-9     # rebalance at every frame end with a moved point
    n = soa.shape[1]
    ref_hist, ref_full = one_partition(prms, soa, PRECISION_FP64)
    with PartitionedSim(prms, n, PRECISION_FP64) as m:
        m.upload(soa)
        hist = m.step(STEPS)
        _, rebalances, _ = m.stats()
        out, ids = m.download()
    assert rebalances > 0
    assert len(ids) == n     # a rebalance drops the disabled slots
    compare(f"3 partitions with {rebalances} rebalances", hist, by_id(out, ids, n), ref_hist, ref_full, True)


def test_overlap_contact_force_counted_once():
    """5 partitions on the block: a slab boundary lies in the indenter's
    contact zone, where both partitions update the overlap nodes."""
    prms, soa = moving_block(5, seed=73, contact=True)
    n = soa.shape[1]
    ref_hist, ref_full = one_partition(prms, soa, PRECISION_FP64, steps=60)
    with PartitionedSim(prms, n, PRECISION_FP64) as m:
        m.upload(soa)
        info = m.info()
        hist = m.step(60)
    r = prms.IndDiameter / 2
    contact = (prms.indenter_x - r) / prms.cellsize, (prms.indenter_x + r + 15.2 * 60 * prms.InitialTimeStep) / prms.cellsize
    bounds = [x0 for x0, _, _, _ in info[1:]]
    assert any(contact[0] - prms.GridHaloSize <= b <= contact[1] + prms.GridHaloSize for b in bounds), (bounds, contact)
    assert np.linalg.norm(ref_hist[:60]) > 0
    e = float(np.linalg.norm(hist - ref_hist[:60]) / np.linalg.norm(ref_hist[:60]))
    print(f"\n5 partitions, contact across a slab boundary: force {e:.2e}")
    assert e < 1e-9, e


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, precision):
    import torch
    import torch.distributed as dist
    from icempm_3dm_b200.partitions import DistTransport, RankPartition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prms, soa = moving_block(world)
        part = RankPartition(prms, soa.shape[1], DistTransport(device=torch.device("cuda", 0)), precision, device=0)
        part.upload(soa)
        hist = part.step(STEPS)
        out, ids = part.download()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), hist=hist, out=out, ids=ids, moved=part.disabled)
        part.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED], ids=["fp64", "mixed"])
def test_one_partition_per_process_matches(precision, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), precision), nprocs=world, join=True)
    prms, soa = moving_block(world)
    n = soa.shape[1]
    ref_hist, ref_full = one_partition(prms, soa, precision)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert np.array_equal(parts[0]["hist"], parts[1]["hist"])     # every rank holds the summed history
    out = np.concatenate([p["out"] for p in parts], axis=1)
    ids = np.concatenate([p["ids"] for p in parts])
    assert sum(int(p["moved"]) for p in parts) > 0
    compare(f"{world} processes ({'fp64' if precision == PRECISION_FP64 else 'mixed'})", parts[0]["hist"],
            by_id(out, ids, n), ref_hist, ref_full, precision == PRECISION_FP64)


def test_bench_partitions_line():
    """bench.py --partitions: one JSON line with the partitioned and the
    one-partition run of the same driver; the FP64 force histories agree."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--workload", "block250k", "--precision",
                        "fp64", "--partitions", "3", "--steps", "20", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["config"]["partitions"] == 3 and line["value"] > 0
    one, many = line["one_partition"]["force_norm"], line["partitioned"]["force_norm"]
    assert one > 0 and abs(many - one) <= 1e-9 * one
