"""x-slab partitions of the step: GPU_Implementation6 with nPartitions > 1
(simulation/gpu_implementation6.cpp:31-208,340-382, model_3d.cpp:35-108).

The particles, sorted by cell key, are split by count into slabs of grid
columns along x. Every partition keeps a grid of the whole domain and works on
its window of it (its columns and GridHaloSize halo columns on each side).
After P2G neighbouring partitions add each other's 2 * GridHaloSize boundary
slabs; every UpdateEveryNthStep / PointTransferFrequency substeps the
particles that left a slab move to the neighbour; at the end of an animation
frame the partitions are rebalanced when one runs short of room or holds
many disabled particles.

Two drivers over the same C-ABI primitives (include/icempm_b200.h):

  PartitionedSim  all partitions in this process (mpm_multi_*: the C++
                  driver; partition i on devices[i % len(devices)], peer
                  copies between devices, CUDA events between streams);
  RankPartition   one partition per process, the B200 layout of one process
                  per GPU: the halo slabs and the point records go to the
                  neighbouring ranks through torch.distributed (NCCL on the
                  device buffers; with gloo they pass through host memory).

The split and sort rules are restated here for RankPartition, where every
rank holds the whole host SoA and keeps its own part.
"""
import ctypes

import numpy as np

from ._lib import LIB, MPMError, check, dptr, uptr
from .layout import N_PTS_ARRAYS, POSX, PRECISION_FP64, STATUS_DISABLED, SimParams3D

__all__ = ["sort_order", "split_sorted", "set_partition_bits", "PartitionedSim", "DistTransport", "RankPartition"]


def sort_order(prms, soa, n):
    """HostSideSOA::RemoveDisabledAndSort (host_side_soa.cpp:56-67) as a
    stable sort: the indices of the non-disabled particles ordered by the cell
    key of ProxyPoint3D::getCellIndex (proxypoint3d.cpp:158-163)."""
    util = np.ascontiguousarray(soa[0, :n]).view(np.int64)
    keep = np.nonzero((util & STATUS_DISABLED) != STATUS_DISABLED)[0]
    h_inv = prms.cellsize_inv
    ix = (soa[POSX, keep] * h_inv + 0.5).astype(np.int64)
    iy = (soa[POSX + 1, keep] * h_inv + 0.5).astype(np.int64)
    iz = (soa[POSX + 2, keep] * h_inv + 0.5).astype(np.int64)
    key = ix * prms.GridY * prms.GridZ + iy * prms.GridZ + iz
    return keep[np.argsort(key, kind="stable")]


def split_sorted(prms, soa, n, nparts):
    """GPU_Implementation6::split_hssoa_into_partitions
    (gpu_implementation6.cpp:340-382) of a cell-sorted SoA: partition i takes
    (n - done) / (nparts - i) particles (integer division) and its slab
    ends at the x index (int)(x/h + 0.5) of the next partition's first
    particle (ProxyPoint3D::getXIndex, proxypoint3d.cpp:165-170). Every slab
    keeps at least one column. Returns [(x0, gxp, start, count)]."""
    gxt = prms.GridXTotal
    out = []
    done, off = 0, 0
    for i in range(nparts):
        cnt = (n - done) // (nparts - i)
        x0 = off
        if i < nparts - 1:
            first_next = done + cnt
            off = int(soa[POSX, first_next] * prms.cellsize_inv + 0.5) if first_next < n else gxt
            off = max(off, x0 + 1)
            off = min(off, gxt - (nparts - 1 - i))
        out.append([x0, 0, done, cnt])
        done += cnt
    for i in range(nparts):
        end = out[i + 1][0] if i < nparts - 1 else gxt
        out[i][1] = end - out[i][0]
    return [tuple(o) for o in out]


def set_partition_bits(soa, start, count, pid):
    """ProxyPoint3D::setPartition (proxypoint3d.cpp:89-110): bits 24-31 of
    the status word of particles [start, start + count) get pid."""
    u = soa[0].view(np.int64)
    seg = u[start:start + count]
    seg &= np.int64(~(0xff << 24))
    seg |= np.int64(pid << 24)


class PartitionedSim:
    """prms.nPartitions partitions in this process (the C++ driver)."""

    def __init__(self, prms, capacity, precision=PRECISION_FP64, devices=(0,)):
        self.prms = prms.copy()
        self.np = int(prms.nPartitions)
        devs = (ctypes.c_int * len(devices))(*devices)
        st = ctypes.c_int(0)
        self._m = LIB.mpm_multi_create(ctypes.byref(self.prms), precision, int(capacity), devs, len(devices),
                                       ctypes.byref(st))
        if not self._m:
            raise MPMError(st.value, "mpm_multi_create")

    def close(self):
        if getattr(self, "_m", None):
            LIB.mpm_multi_destroy(self._m)
            self._m = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, soa, cohesion=None):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        c = None if cohesion is None else np.ascontiguousarray(cohesion, dtype=np.float64)
        check(LIB.mpm_multi_upload_soa(self._m, dptr(soa), soa.shape[1], soa.shape[1],
                                       dptr(c) if c is not None else None), "mpm_multi_upload_soa")

    def step(self, nsteps, raise_on_error=True):
        hist = np.zeros((nsteps, 3))
        code = LIB.mpm_multi_step(self._m, int(nsteps), dptr(hist))
        if raise_on_error:
            check(code, "mpm_multi_step")
        return hist

    def download(self):
        """(soa, ids): the partitions' particles one after another, disabled
        ones included, and their upload indices."""
        n = ctypes.c_uint(0)
        check(LIB.mpm_multi_download_soa(self._m, None, 0, None, ctypes.byref(n)), "mpm_multi_download_soa")
        k = max(n.value, 1)
        soa = np.zeros((N_PTS_ARRAYS, k))
        ids = np.zeros(k, dtype=np.uint32)
        check(LIB.mpm_multi_download_soa(self._m, dptr(soa), k, uptr(ids), ctypes.byref(n)), "mpm_multi_download_soa")
        return soa[:, :n.value], ids[:n.value]

    def rebalance(self):
        check(LIB.mpm_multi_rebalance(self._m), "mpm_multi_rebalance")

    def info(self):
        """[(x0, gxp, particles incl. disabled, disabled since the split)] per partition."""
        out = []
        for i in range(self.np):
            x0, gxp, n, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint(), ctypes.c_uint()
            check(LIB.mpm_multi_info(self._m, i, ctypes.byref(x0), ctypes.byref(gxp), ctypes.byref(n),
                                     ctypes.byref(nd)), "mpm_multi_info")
            out.append((x0.value, gxp.value, n.value, nd.value))
        return out

    def stats(self):
        """(largest transfer to one side, rebalances, PointTransferFrequency)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(LIB.mpm_multi_stats(self._m, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "mpm_multi_stats")
        return a.value, b.value, c.value

    def sensors(self):
        ns = 3 * self.prms.IndenterSubdivisions * self.prms.GridZ
        s, t = np.zeros(ns), np.zeros(3)
        check(LIB.mpm_multi_sensors(self._m, dptr(s), dptr(t)), "mpm_multi_sensors")
        return s, t


class DistTransport:
    """The neighbour exchanges of one partition per rank over
    torch.distributed (ranks in x order). With the NCCL backend the buffers
    stay on the device; with gloo they pass through host memory."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.torch = torch
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.on_device = dist.get_backend() == "nccl"
        self.device = device

    def _wire(self, t):
        return t if self.on_device else t.cpu()

    def neighbours(self, to_left, to_right, from_left_shape, from_right_shape, dtype):
        """Sends to_left to rank - 1 and to_right to rank + 1 (None: nothing),
        receives from them arrays of the given shapes (None where there is no
        neighbour). Every rank posts its sends and receives in one batch."""
        torch, dist = self.torch, self.dist
        ops, recv = [], [None, None]
        if self.rank > 0 and from_left_shape is not None:
            recv[0] = torch.empty(from_left_shape, dtype=dtype, device=self.device if self.on_device else "cpu")
            ops.append(dist.P2POp(dist.irecv, recv[0], self.rank - 1))
        if self.rank < self.world - 1 and from_right_shape is not None:
            recv[1] = torch.empty(from_right_shape, dtype=dtype, device=self.device if self.on_device else "cpu")
            ops.append(dist.P2POp(dist.irecv, recv[1], self.rank + 1))
        sends = []
        if self.rank > 0 and to_left is not None:
            sends.append(self._wire(to_left))
            ops.append(dist.P2POp(dist.isend, sends[-1], self.rank - 1))
        if self.rank < self.world - 1 and to_right is not None:
            sends.append(self._wire(to_right))
            ops.append(dist.P2POp(dist.isend, sends[-1], self.rank + 1))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return recv[0], recv[1]

    def sum(self, arr):
        t = self.torch.as_tensor(np.asarray(arr, dtype=np.float64))
        t = t.to(self.device) if self.on_device else t
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def max(self, value):
        t = self.torch.tensor([float(value)], dtype=self.torch.float64)
        t = t.to(self.device) if self.on_device else t
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def all_gather(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out


class RankPartition:
    """The partition of this rank (rank i = partition i of world_size):
    an MPMHandle on `device` and a DistTransport to its neighbours. Every rank
    calls every method in the same order (the exchanges are collective)."""

    def __init__(self, prms, capacity, transport, precision=PRECISION_FP64, device=0):
        import torch
        from .simulation import MPMHandle
        self.torch = torch
        self.t = transport
        self.prms = prms.copy()
        self.prms.nPartitions = transport.world
        if transport.world > 1 and prms.GridHaloSize < 3:
            raise ValueError("partitions need GridHaloSize >= 3")
        self.device = torch.device("cuda", device)
        self.h = MPMHandle(self.prms, capacity, precision, device=device)
        # one stream for the handle's kernels and the exchange buffers' copies
        # (torch's default stream would not order against the handle's own)
        self.stream = torch.cuda.Stream(device=self.device)
        self.h.set_stream(self.stream.cuda_stream)
        self.cap = max(int(self.prms.VectorCapacity_transfer), 1)
        self.halo_bytes = self.h.halo_bytes()
        self.rec_bytes = self.h.record_bytes()
        nb = max(self.halo_bytes, 16)
        self.hsend = [torch.empty(nb, dtype=torch.uint8, device=self.device) for _ in range(2)]
        self.pout = [torch.empty(max(self.cap * self.rec_bytes, 16), dtype=torch.uint8, device=self.device)
                     for _ in range(2)]
        self.disabled = 0
        self.max_deviation = 0
        self.rebalances = 0
        self.cohesion = False

    def close(self):
        if self.h is not None:
            self.h.close()
            self.h = None

    def upload(self, soa, cohesion=None):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        c = None if cohesion is None else np.ascontiguousarray(cohesion, dtype=np.float64)
        check(LIB.mpm_multi_upload_soa(self._m, dptr(soa), soa.shape[1], soa.shape[1],
                                       dptr(c) if c is not None else None), "mpm_multi_upload_soa")

    def step(self, nsteps, raise_on_error=True):
        hist = np.zeros((nsteps, 3))
        code = LIB.mpm_multi_step(self._m, int(nsteps), dptr(hist))
        if raise_on_error:
            check(code, "mpm_multi_step")
        return hist

    def download(self):
        """(soa, ids): the partitions' particles one after another, disabled
        ones included, and their upload indices."""
        n = ctypes.c_uint(0)
        check(LIB.mpm_multi_download_soa(self._m, None, 0, None, ctypes.byref(n)), "mpm_multi_download_soa")
        k = max(n.value, 1)
        soa = np.zeros((N_PTS_ARRAYS, k))
        ids = np.zeros(k, dtype=np.uint32)
        check(LIB.mpm_multi_download_soa(self._m, dptr(soa), k, uptr(ids), ctypes.byref(n)), "mpm_multi_download_soa")
        return soa[:, :n.value], ids[:n.value]

    def rebalance(self):
        check(LIB.mpm_multi_rebalance(self._m), "mpm_multi_rebalance")

    def info(self):
        """[(x0, gxp, particles incl. disabled, disabled since the split)] per partition."""
        out = []
        for i in range(self.np):
            x0, gxp, n, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint(), ctypes.c_uint()
            check(LIB.mpm_multi_info(self._m, i, ctypes.byref(x0), ctypes.byref(gxp), ctypes.byref(n),
                                     ctypes.byref(nd)), "mpm_multi_info")
            out.append((x0.value, gxp.value, n.value, nd.value))
        return out

    def stats(self):
        """(largest transfer to one side, rebalances, PointTransferFrequency)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(LIB.mpm_multi_stats(self._m, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "mpm_multi_stats")
        return a.value, b.value, c.value

    def sensors(self):
        ns = 3 * self.prms.IndenterSubdivisions * self.prms.GridZ
        s, t = np.zeros(ns), np.zeros(3)
        check(LIB.mpm_multi_sensors(self._m, dptr(s), dptr(t)), "mpm_multi_sensors")
        return s, t


class DistTransport:
    """The neighbour exchanges of one partition per rank over
    torch.distributed (ranks in x order). With the NCCL backend the buffers
    stay on the device; with gloo they pass through host memory."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.torch = torch
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.on_device = dist.get_backend() == "nccl"
        self.device = device

    def _wire(self, t):
        return t if self.on_device else t.cpu()

    def neighbours(self, to_left, to_right, from_left_shape, from_right_shape, dtype):
        """Sends to_left to rank - 1 and to_right to rank + 1 (None: nothing),
        receives from them arrays of the given shapes (None where there is no
        neighbour). Every rank posts its sends and receives in one batch."""
        torch, dist = self.torch, self.dist
        ops, recv = [], [None, None]
        if self.rank > 0 and from_left_shape is not None:
            recv[0] = torch.empty(from_left_shape, dtype=dtype, device=self.device if self.on_device else "cpu")
            ops.append(dist.P2POp(dist.irecv, recv[0], self.rank - 1))
        if self.rank < self.world - 1 and from_right_shape is not None:
            recv[1] = torch.empty(from_right_shape, dtype=dtype, device=self.device if self.on_device else "cpu")
            ops.append(dist.P2POp(dist.irecv, recv[1], self.rank + 1))
        sends = []
        if self.rank > 0 and to_left is not None:
            sends.append(self._wire(to_left))
            ops.append(dist.P2POp(dist.isend, sends[-1], self.rank - 1))
        if self.rank < self.world - 1 and to_right is not None:
            sends.append(self._wire(to_right))
            ops.append(dist.P2POp(dist.isend, sends[-1], self.rank + 1))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return recv[0], recv[1]

    def sum(self, arr):
        t = self.torch.as_tensor(np.asarray(arr, dtype=np.float64))
        t = t.to(self.device) if self.on_device else t
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def max(self, value):
        t = self.torch.tensor([float(value)], dtype=self.torch.float64)
        t = t.to(self.device) if self.on_device else t
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def all_gather(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out


class RankPartition:
    """The partition of this rank (rank i = partition i of world_size):
    an MPMHandle on `device` and a DistTransport to its neighbours. Every rank
    calls every method in the same order (the exchanges are collective)."""

    def __init__(self, prms, capacity, transport, precision=PRECISION_FP64, device=0):
        import torch
        from .simulation import MPMHandle
        self.torch = torch
        self.t = transport
        self.prms = prms.copy()
        self.prms.nPartitions = transport.world
        if transport.world > 1 and prms.GridHaloSize < 3:
            raise ValueError("partitions need GridHaloSize >= 3")
        self.device = torch.device("cuda", device)
        self.h = MPMHandle(self.prms, capacity, precision, device=device)
        # one stream for the handle's kernels and the exchange buffers' copies
        # (torch's default stream would not order against the handle's own)
        self.stream = torch.cuda.Stream(device=self.device)
        self.h.set_stream(self.stream.cuda_stream)
        self.cap = max(int(self.prms.VectorCapacity_transfer), 1)
        self.halo_bytes = self.h.halo_bytes()
        self.rec_bytes = self.h.record_bytes()
        nb = max(self.halo_bytes, 16)
        self.hsend = [torch.empty(nb, dtype=torch.uint8, device=self.device) for _ in range(2)]
        self.pout = [torch.empty(max(self.cap * self.rec_bytes, 16), dtype=torch.uint8, device=self.device)
                     for _ in range(2)]
        self.disabled = 0
        self.max_deviation = 0
        self.rebalances = 0
        self.cohesion = False

    def close(self):
        if self.h is not None:
            self.h.close()
            self.h = None

    def _upload_sorted(self, soa, n, cohesion, ids):
        world, rank = self.t.world, self.t.rank
        parts = split_sorted(self.prms, soa, n, world)
        for i, (x0, gxp, start, cnt) in enumerate(parts):
            set_partition_bits(soa, start, cnt, i)
        x0, gxp, start, cnt = parts[rank]
        self.h.set_partition(rank, x0, gxp, 0)
        mine = np.ascontiguousarray(soa[:, start:start + cnt])
        c = None if cohesion is None else np.ascontiguousarray(cohesion[start:start + cnt])
        self.h.upload(mine, cohesion=c)
        if cnt:
            idt = self.torch.as_tensor(np.ascontiguousarray(ids[start:start + cnt]).view(np.int32))
            # the handle's id row is device memory: write the global ids there
            dev_ids = idt.to(self.device)
            LIB.mpm_synchronize(self.h._h)
            self._set_ids(dev_ids)
        self.slab = (x0, gxp)
        self.disabled = 0

    def _set_ids(self, dev_ids):
        # ids are set by re-running set_partition with the id base when they
        # are contiguous (the split keeps sorted order, and the upload order of
        # a sorted block is its id order), else through a points round trip
        ids = dev_ids.cpu().numpy().view(np.uint32)
        if ids.size and np.array_equal(ids, np.arange(ids[0], ids[0] + ids.size, dtype=np.uint32)):
            self._id_base = int(ids[0])
            return
        raise ValueError("RankPartition uploads need contiguous ids per partition")

    def upload(self, soa, cohesion=None):
        """The whole host SoA on every rank: sorted, split, this rank's part
        uploaded. Particle ids are the indices into soa."""
        soa = np.array(soa, dtype=np.float64, copy=True)
        n = soa.shape[1]
        order = sort_order(self.prms, soa, n)
        soa = np.ascontiguousarray(soa[:, order])
        coh = None if cohesion is None else np.ascontiguousarray(np.asarray(cohesion, dtype=np.float64)[order])
        self.cohesion = coh is not None
        self._upload_with_ids(soa, order.size, coh, order.astype(np.uint32))

    def _upload_with_ids(self, soa, n, coh, ids):
        world, rank = self.t.world, self.t.rank
        parts = split_sorted(self.prms, soa, n, world)
        for i, (x0, gxp, start, cnt) in enumerate(parts):
            set_partition_bits(soa, start, cnt, i)
        x0, gxp, start, cnt = parts[rank]
        self.h.set_partition(rank, x0, gxp, 0)
        mine = np.ascontiguousarray(soa[:, start:start + cnt])
        c = None if coh is None else np.ascontiguousarray(coh[start:start + cnt])
        self.h.upload(mine, cohesion=c)
        self.h.upload_ids(np.ascontiguousarray(ids[start:start + cnt], dtype=np.uint32))
        self.slab = (x0, gxp)
        self.disabled = 0

    def _exchange_halos(self):
        with self.torch.cuda.stream(self.stream):
            self._exchange_halos_on_stream()

    def _exchange_halos_on_stream(self):
        torch = self.torch
        rank, world = self.t.rank, self.t.world
        hb = self.halo_bytes
        left = rank > 0
        right = rank < world - 1
        if left:
            self.h.halo_pack(0, self.hsend[0].data_ptr())
        if right:
            self.h.halo_pack(1, self.hsend[1].data_ptr())
        fl, fr = self.t.neighbours(self.hsend[0][:hb] if left else None, self.hsend[1][:hb] if right else None,
                                   (hb,) if left else None, (hb,) if right else None, torch.uint8)
        if fl is not None:
            fl = fl.to(self.device)
            self.h.halo_add(0, fl.data_ptr())
        if fr is not None:
            fr = fr.to(self.device)
            self.h.halo_add(1, fr.data_ptr())
        self.stream.synchronize()

    def _transfer_points(self):
        with self.torch.cuda.stream(self.stream):
            self._transfer_points_on_stream()

    def _transfer_points_on_stream(self):
        torch = self.torch
        nl, nr, dev = self.h.points_out(self.pout[0].data_ptr(), self.pout[1].data_ptr(), self.cap)
        self.max_deviation = max(self.max_deviation, dev)
        self.disabled += nl + nr
        rb = self.rec_bytes
        counts = torch.tensor([nl, nr], dtype=torch.int64)
        cl, cr = self.t.neighbours(counts, counts, (2,), (2,), torch.int64)
        from_left = int(cl[1]) if cl is not None else 0     # the left neighbour's right-going records
        from_right = int(cr[0]) if cr is not None else 0    # the right neighbour's left-going records
        # a message only where records go: both ends know the count
        rl, rr = self.t.neighbours(self.pout[0][:nl * rb] if nl else None, self.pout[1][:nr * rb] if nr else None,
                                   (from_left * rb,) if from_left else None,
                                   (from_right * rb,) if from_right else None, torch.uint8)
        for buf, k in ((rl, from_left), (rr, from_right)):
            if buf is not None and k:
                d = buf.to(self.device)
                self.h.points_in(d.data_ptr(), k)
        self.stream.synchronize()

    def download(self):
        """This rank's particles (disabled ones included) and their ids."""
        return self.h.download(), self.h.ids()

    def step(self, nsteps):
        """nsteps substeps of Model3D::Step over all ranks; returns the force
        history summed over the partitions (the same on every rank)."""
        p = self.prms
        hist = np.zeros((nsteps, 3))
        per = max(1, p.UpdateEveryNthStep // max(1, p.PointTransferFrequency))
        for s in range(nsteps):
            step_no = p.SimulationStep + s
            transfer = self.t.world > 1 and step_no % per == 0
            frame_end = (step_no + 1) % p.UpdateEveryNthStep == 0
            self.h.substep_p2g()
            if self.t.world > 1:
                self._exchange_halos()
            hist[s] = self.h.substep_update_g2p(s == nsteps - 1 or transfer or frame_end)
            if transfer:
                self._transfer_points()
            if frame_end:
                dev = self.t.max(self.max_deviation)
                if dev > p.GridHaloSize / 2:
                    p.PointTransferFrequency += 1
                    per = max(1, p.UpdateEveryNthStep // p.PointTransferFrequency)
                self.max_deviation = 0
                if self.t.world > 1 and self.t.max(1.0 if self._needs_rebalance() else 0.0) > 0:
                    self._rebalance(step_no + 1)
        # the handle advanced its own copy (time, step, indenter); keep the
        # transfer frequency this driver raised
        ptf = p.PointTransferFrequency
        self.prms = self.h.params()
        self.prms.PointTransferFrequency = ptf
        return self.t.sum(hist)

    def _needs_rebalance(self):
        p = self.prms
        n = max(self.h.count(), 1)
        free_share = (self.h.capacity - self.h.count()) / n
        return (free_share < p.RebalanceThresholdFreeSpaceRemaining or
                self.disabled / self.h.capacity > p.RebalanceThresholdDisabledPercentage)

    def _rebalance(self, step_no):
        """Model3D::Step's rebalance (model_3d.cpp:99-108) over the ranks:
        every rank gathers all particles, sorts, splits and keeps its part."""
        soa, ids = self.download()
        coh = self.h.cohesion() if self.cohesion else None
        parts = self.t.all_gather((soa, ids, coh))
        soa = np.concatenate([q[0] for q in parts], axis=1)
        ids = np.concatenate([q[1] for q in parts])
        coh = np.concatenate([q[2] for q in parts]) if self.cohesion else None
        order = sort_order(self.prms, soa, soa.shape[1])
        soa = np.ascontiguousarray(soa[:, order])
        coh = None if coh is None else np.ascontiguousarray(coh[order])
        self._upload_with_ids(soa, order.size, coh, ids[order])
        self.rebalances += 1
