"""Host logic of the x-slab partitions (icempm_3dm_b200.partitions), on CPU:
the sort and split rules against the reference's, and the neighbour
exchanges of one partition per rank over torch.distributed with gloo ranks
(world sizes 2 and 3)."""
import os
import socket

import numpy as np
import pytest

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200.layout import IDX_UTILITY, POSX, STATUS_DISABLED
from icempm_3dm_b200.partitions import set_partition_bits, sort_order, split_sorted
from oracle import params as oracle_params
from oracle import pyoracle as po
from tests.helpers import util_as_double, util_bits


def reference_split(hinv, gxt, xs, n, nparts):
    """split_hssoa_into_partitions (gpu_implementation6.cpp:340-382) as
    written: the count of partition i, GridX_offset and GridX_partition."""
    processed, out, offsets = 0, [], [0] * nparts
    for i in range(nparts):
        npts = (n - processed) // (nparts - i)
        if i < nparts - 1:
            cells = int(xs[processed + npts] * hinv + 0.5)      # getXIndex of the next partition's first point
            gxp = cells - offsets[i]
            offsets[i + 1] = cells
        else:
            gxp = gxt - offsets[i]
        out.append((offsets[i], gxp, processed, npts))
        processed += npts
    return out


@pytest.mark.parametrize("nparts", [1, 2, 3, 5])
def test_split_matches_the_reference(nparts):
    prms, soa, _ = gen.small_block(n=5000, seed=61, dims=(0.4, 0.1, 0.1), ops=oracle_params.OPS)
    n = soa.shape[1]
    order = sort_order(prms, soa, n)
    s = np.ascontiguousarray(soa[:, order])
    got = split_sorted(prms, s, n, nparts)
    ref = reference_split(prms.cellsize_inv, prms.GridXTotal, s[POSX], n, nparts)
    assert got == ref
    assert sum(c for _, _, _, c in got) == n
    assert all(g >= 1 for _, g, _, _ in got)


def test_sort_order_is_the_oracles_stable_sort():
    prms, soa, _ = gen.small_block(n=4000, seed=62, ops=oracle_params.OPS)
    n = soa.shape[1]
    rng = np.random.default_rng(62)
    soa = np.ascontiguousarray(soa[:, rng.permutation(n)])
    bits = util_bits(soa).copy()
    bits[rng.random(n) < 0.1] |= STATUS_DISABLED
    soa[IDX_UTILITY] = util_as_double(bits)
    soa[POSX:POSX + 3, 1:200:2] = soa[POSX:POSX + 3, 0:199:2]     # ties
    assert np.array_equal(sort_order(prms, soa, n), po.sort_permutation(prms, soa, n))


def test_partition_bits():
    soa = np.zeros((28, 10))
    bits = np.full(10, 0x12345 | (0x7f << 24) | (1 << 40), dtype=np.int64)
    soa[IDX_UTILITY] = util_as_double(bits)
    set_partition_bits(soa, 2, 5, 9)
    b = util_bits(soa)
    assert np.all((b[2:7] >> 24) & 0xff == 9) and np.all((b[:2] >> 24) & 0xff == 0x7f)
    assert np.all(b & 0xffffff == 0x12345) and np.all(b >> 40 == 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    from icempm_3dm_b200.partitions import DistTransport
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = DistTransport()
        # halos: rank r sends [r*10 + 1] * (r + 3) bytes left and [r*10 + 2] * (r + 4) right
        to_l = torch.full((rank + 3,), rank * 10 + 1, dtype=torch.uint8)
        to_r = torch.full((rank + 4,), rank * 10 + 2, dtype=torch.uint8)
        fl, fr = t.neighbours(to_l, to_r, (rank - 1 + 4,) if rank > 0 else None,
                              (rank + 1 + 3,) if rank < world - 1 else None, torch.uint8)
        # records: only where the sender has some (rank r sends r to the right, none to the left)
        cnt = torch.tensor([0, rank], dtype=torch.int64)
        cl, cr = t.neighbours(cnt, cnt, (2,), (2,), torch.int64)
        from_left = int(cl[1]) if cl is not None else 0
        rec = torch.arange(rank, dtype=torch.float64) + 100 * rank
        rl, rr = t.neighbours(None, rec if rank else None, (from_left,) if from_left else None, None, torch.float64)
        s = t.sum(np.array([rank + 1.0, 2.0]))
        m = t.max(rank * 3)
        g = t.all_gather(("rank", rank))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"),
                 fl=fl.numpy() if fl is not None else np.zeros(0), fr=fr.numpy() if fr is not None else np.zeros(0),
                 rl=rl.numpy() if rl is not None else np.zeros(0), s=s, m=m, g=np.array([x[1] for x in g]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_neighbour_exchanges_over_gloo(world, tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        z = np.load(tmp_path / f"r{r}.npz")
        if r > 0:    # from the left: its right-going halo
            assert np.array_equal(z["fl"], np.full(r - 1 + 4, (r - 1) * 10 + 2, dtype=np.uint8))
            assert np.array_equal(z["rl"], np.arange(r - 1) + 100.0 * (r - 1))
        else:
            assert z["fl"].size == 0 and z["rl"].size == 0
        if r < world - 1:
            assert np.array_equal(z["fr"], np.full(r + 1 + 3, (r + 1) * 10 + 1, dtype=np.uint8))
        else:
            assert z["fr"].size == 0
        assert np.allclose(z["s"], [world * (world + 1) / 2, 2.0 * world])
        assert float(z["m"]) == 3.0 * (world - 1)
        assert list(z["g"]) == list(range(world))
