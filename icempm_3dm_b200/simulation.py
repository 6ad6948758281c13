"""Host-side mirror of the reference's step API over the C-ABI.

  MPMHandle            one partition on one GPU (mpm_create ... mpm_destroy)
  GPU_Implementation6  the reference class's method names and call order
                       (simulation/gpu_implementation6.h:24-59) for one
                       partition: halo and point-transfer methods are no-ops
  Model3D              the substep loop of Model3D::Step (model_3d.cpp:24-112)
  SnapshotManager      raw point-cloud loading, full snapshots and resume
                       (snapshotmanager.cpp:20-113, :299-405) in the
                       reference's HDF5 layout

All device work runs in the CUDA library; nothing here computes physics.
"""
import ctypes
import os

import numpy as np

from . import snapshot as _snap
from ._lib import (LIB, N_PTS_ARRAYS, PRECISION_FP64, MPMError, SimParams3D, check, dptr, uptr)


class MPMHandle:
    def __init__(self, prms, capacity, precision=PRECISION_FP64, device=0):
        st = ctypes.c_int(0)
        self.prms = prms.copy()
        self.precision = precision
        self._h = LIB.mpm_create(ctypes.byref(self.prms), precision, int(capacity), device, ctypes.byref(st))
        if not self._h:
            raise MPMError(st.value, "mpm_create")
        self.capacity = int(capacity)
        self._adj_steps = None   # substeps of the last adjoint_forward

    def close(self):
        if getattr(self, "_h", None):
            LIB.mpm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data
    def upload(self, soa, n=None, cohesion=None):
        soa = np.ascontiguousarray(soa, dtype=np.float64)
        if soa.ndim != 2 or soa.shape[0] != N_PTS_ARRAYS:
            raise ValueError(f"soa must have shape ({N_PTS_ARRAYS}, pitch), got {soa.shape}")
        n = soa.shape[1] if n is None else int(n)
        if not 0 <= n <= soa.shape[1]:
            raise ValueError(f"n = {n} outside 0..{soa.shape[1]} (the soa's pitch)")
        c = None
        if cohesion is not None:
            c = np.ascontiguousarray(cohesion, dtype=np.float64).ravel()
            if c.size < n:
                raise ValueError(f"cohesion holds {c.size} values for {n} particles")
        check(LIB.mpm_upload_soa(self._h, dptr(soa), soa.shape[1], n), "mpm_upload_soa")
        if c is not None:
            check(LIB.mpm_upload_cohesion(self._h, dptr(c), n), "mpm_upload_cohesion")

    def count(self):
        n = ctypes.c_uint(0)
        check(LIB.mpm_count(self._h, ctypes.byref(n)), "mpm_count")
        return n.value

    def download(self, raise_on_error=True, out=None):
        """mpm_download_soa: the particles as a (28, n) SoA. out: a
        C-contiguous float64 array of 28 rows and at least n columns (e.g.
        from pinned_empty, which copies at the host link's speed) that
        receives them; the view out[:, :n] is returned."""
        n = self.count()
        if out is None:
            soa = np.zeros((N_PTS_ARRAYS, max(n, 1)), dtype=np.float64)
        else:
            if (out.dtype != np.float64 or out.ndim != 2 or out.shape[0] != N_PTS_ARRAYS
                    or not out.flags.c_contiguous or out.shape[1] < max(n, 1)):
                raise ValueError(f"out must be a C-contiguous float64 array of {N_PTS_ARRAYS} rows and at least "
                                 f"{max(n, 1)} columns")
            soa = out
        nn = ctypes.c_uint(0)
        code = LIB.mpm_download_soa(self._h, dptr(soa), soa.shape[1], ctypes.byref(nn))
        if raise_on_error:
            check(code, "mpm_download_soa")
        return soa[:, :nn.value]

    def ids(self):
        n = self.count()
        ids = np.zeros(max(n, 1), dtype=np.uint32)
        nn = ctypes.c_uint(0)
        check(LIB.mpm_download_ids(self._h, uptr(ids), ctypes.byref(nn)), "mpm_download_ids")
        return ids[:nn.value]

    def sort(self):
        return check(LIB.mpm_sort(self._h), "mpm_sort")

    def set_grid_accumulation(self, mode):
        """ACCUM_FLOAT (default) or ACCUM_FIXED (mixed handles: order-
        independent fixed-point grid sums, runs repeat bit for bit)."""
        check(LIB.mpm_set_grid_accumulation(self._h, int(mode)), "mpm_set_grid_accumulation")

    def upload_ids(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        check(LIB.mpm_upload_ids(self._h, uptr(ids), ids.size), "mpm_upload_ids")

    def cohesion(self):
        n = self.count()
        c = np.zeros(max(n, 1))
        nn = ctypes.c_uint(0)
        check(LIB.mpm_download_cohesion(self._h, dptr(c), ctypes.byref(nn)), "mpm_download_cohesion")
        return c[:nn.value]

    # -- x-slab partition (one partition of a partitioned run)
    def set_partition(self, pid, x0, gxp, id_base=0):
        check(LIB.mpm_set_partition(self._h, int(pid), int(x0), int(gxp), int(id_base)), "mpm_set_partition")

    def halo_bytes(self):
        return int(LIB.mpm_halo_bytes(self._h))

    def halo_pack(self, side, dst_ptr):
        check(LIB.mpm_halo_pack(self._h, int(side), ctypes.c_void_p(dst_ptr)), "mpm_halo_pack")

    def halo_add(self, side, src_ptr):
        check(LIB.mpm_halo_add(self._h, int(side), ctypes.c_void_p(src_ptr)), "mpm_halo_add")

    def record_bytes(self):
        return int(LIB.mpm_point_record_bytes(self._h))

    def points_out(self, left_ptr, right_ptr, capacity):
        """(records to the left, to the right, max deviation in columns)."""
        nl, nr, dev = ctypes.c_uint(0), ctypes.c_uint(0), ctypes.c_int(0)
        check(LIB.mpm_points_out(self._h, ctypes.c_void_p(left_ptr), ctypes.c_void_p(right_ptr), int(capacity),
                                 ctypes.byref(nl), ctypes.byref(nr), ctypes.byref(dev)), "mpm_points_out")
        return nl.value, nr.value, dev.value

    def points_in(self, src_ptr, count):
        check(LIB.mpm_points_in(self._h, ctypes.c_void_p(src_ptr), int(count)), "mpm_points_in")

    def substep_p2g(self):
        check(LIB.mpm_substep_p2g(self._h), "mpm_substep_p2g")

    def substep_update_g2p(self, store_vc, want_force=True):
        f = np.zeros(3)
        check(LIB.mpm_substep_update_g2p(self._h, int(store_vc), dptr(f) if want_force else None),
              "mpm_substep_update_g2p")
        return f

    def frame_records(self, frame, full):
        """mpm_frame_records: the VisualPoint records (full) or the
        (UpdatePos, UpdateJp, UpdateStatus) records of this frame."""
        cap = max(self.count(), 1)
        if full:
            pts = np.zeros(cap, dtype=_snap.VISUAL_POINT)
            n = ctypes.c_uint(0)
            check(LIB.mpm_frame_records(self._h, frame, 1, pts.ctypes.data, ctypes.byref(n), None, None, None, None,
                                        None, None), "mpm_frame_records")
            return pts[:n.value]
        pv, jp, st = (np.zeros(cap, dtype=d) for d in (_snap.UPDATE_POS, _snap.UPDATE_JP, _snap.UPDATE_STATUS))
        c = [ctypes.c_uint(0) for _ in range(3)]
        check(LIB.mpm_frame_records(self._h, frame, 0, None, None, pv.ctypes.data, ctypes.byref(c[0]), jp.ctypes.data,
                                    ctypes.byref(c[1]), st.ctypes.data, ctypes.byref(c[2])), "mpm_frame_records")
        return pv[:c[0].value], jp[:c[1].value], st[:c[2].value]

    def set_sort_interval(self, k):
        check(LIB.mpm_set_sort_interval(self._h, k), "mpm_set_sort_interval")

    def update_constants(self, prms=None):
        if prms is not None:
            self.prms = prms.copy()
        check(LIB.mpm_update_constants(self._h, ctypes.byref(self.prms)), "mpm_update_constants")

    def set_stream(self, stream_ptr):
        check(LIB.mpm_set_stream(self._h, ctypes.c_void_p(stream_ptr)), "mpm_set_stream")

    # -- stepping
    def step(self, nsteps, want_forces=True, raise_on_error=True):
        hist = np.zeros((nsteps, 3)) if want_forces else None
        code = LIB.mpm_step(self._h, nsteps, dptr(hist) if want_forces else None)
        if raise_on_error:
            check(code, "mpm_step")
        return hist if want_forces else code

    def params(self):
        out = SimParams3D()
        check(LIB.mpm_get_params(self._h, ctypes.byref(out)), "mpm_get_params")
        return out

    def sensors(self):
        p = self.params()
        s = np.zeros(3 * p.IndenterSubdivisions * p.GridZ)
        tot = np.zeros(3)
        check(LIB.mpm_sensors(self._h, dptr(s), dptr(tot)), "mpm_sensors")
        return s, tot

    def error(self):
        return LIB.mpm_get_error(self._h)

    def synchronize(self):
        check(LIB.mpm_synchronize(self._h), "mpm_synchronize")

    # -- phases (GPU_Implementation6 one-partition subset)
    def reset_grid(self):
        check(LIB.mpm_reset_grid(self._h), "mpm_reset_grid")

    def p2g(self):
        check(LIB.mpm_p2g(self._h), "mpm_p2g")

    def update_nodes(self, ind_x, ind_y):
        check(LIB.mpm_update_nodes(self._h, ind_x, ind_y), "mpm_update_nodes")

    def g2p(self, record_pq):
        check(LIB.mpm_g2p(self._h, int(bool(record_pq))), "mpm_g2p")

    def reset_indenter_force_accumulator(self):
        check(LIB.mpm_reset_indenter_force_accumulator(self._h), "mpm_reset_indenter_force_accumulator")

    def grid(self, which=0):
        p = self.prms
        nodes = (p.GridXTotal + 2 * p.GridHaloSize) * p.GridY * p.GridZ
        g = np.zeros((4, nodes))
        check(LIB.mpm_testing_download_grid(self._h, dptr(g), which), "mpm_testing_download_grid")
        return g

    def step_timed(self, nsteps):
        ms = (ctypes.c_float * 4)()
        check(LIB.mpm_testing_step_timed(self._h, nsteps, ms), "mpm_testing_step_timed")
        return [ms[k] for k in range(4)]

    def active_nodes(self):
        c = ctypes.c_longlong(0)
        check(LIB.mpm_testing_active_nodes(self._h, ctypes.byref(c)), "mpm_testing_active_nodes")
        return c.value

    # -- adjoint (FP64 handles)
    def adjoint_forward(self, nsteps, ckpt_every):
        """nsteps substeps with a device checkpoint every ckpt_every; returns
        the (nsteps, 3) indenter force history."""
        hist = np.zeros((nsteps, 3))
        self._adj_steps = None
        check(LIB.mpm_adjoint_forward(self._h, nsteps, ckpt_every, dptr(hist)), "mpm_adjoint_forward")
        self._adj_steps = int(nsteps)
        return hist

    def adjoint_backward(self, dL_dforce):
        """Reverse sweep for dL/d(force history); returns (dL/dcohesion per
        particle in the handle's order, dL/dYoungsModulus)."""
        g = np.ascontiguousarray(dL_dforce, dtype=np.float64).reshape(-1, 3)
        if self._adj_steps is None:
            raise MPMError(108, "mpm_adjoint_backward before a successful adjoint_forward")   # MPM_ERR_STATE
        if g.shape[0] != self._adj_steps:
            raise ValueError(f"dL_dforce has {g.shape[0]} rows for {self._adj_steps} substeps")
        dc = np.zeros(max(self.count(), 1))
        dE = ctypes.c_double(0.0)
        check(LIB.mpm_adjoint_backward(self._h, dptr(g), dptr(dc), ctypes.byref(dE)), "mpm_adjoint_backward")
        return dc[:self.count()], dE.value

    def adjoint_state(self):
        """(25, n) adjoints of the initial state: x(3), v(3), C(9), F(9), Jp_inv."""
        n = self.count()
        adj = np.zeros((25, max(n, 1)))
        check(LIB.mpm_adjoint_state(self._h, dptr(adj), adj.shape[1]), "mpm_adjoint_state")
        return adj[:, :n]


def pinned_empty(shape, dtype=np.float64):
    """An uninitialised array over page-locked host memory (mpm_host_alloc,
    the memory HostSideSOA::Allocate takes, host_side_soa.cpp:70-86): copies
    between it and the device run at the host link's speed. The memory is
    released (mpm_host_free) when the last array over it is gone."""
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    if nbytes == 0:
        return np.empty(shape, dtype=dtype)
    ptr = ctypes.c_void_p()
    check(LIB.mpm_host_alloc(nbytes, ctypes.byref(ptr)), "mpm_host_alloc")
    free = LIB.mpm_host_free          # bound now: module globals may be gone when the last view dies

    class PinnedBytes(ctypes.c_char * nbytes):
        def __del__(self):
            try:
                free(ctypes.c_void_p(ctypes.addressof(self)))
            except Exception:         # interpreter shutdown: the process returns the memory
                pass

    return np.frombuffer(PinnedBytes.from_address(ptr.value), dtype=dtype).reshape(shape)


class GPU_Implementation6:
    """Method-for-method mirror of the reference class for one partition.
    transfer_from_device downloads into one page-locked host buffer of the
    handle's capacity, reused from frame to frame as the reference reuses
    HostSideSOA's buffer: hssoa is a view of it, overwritten by the next
    transfer."""

    def __init__(self, prms, precision=PRECISION_FP64, device=0):
        self.prms = prms
        self.precision = precision
        self.device = device
        self.handle = None
        self.hssoa = None
        self.indenter_force = np.zeros(3)
        self.indenter_sensor_total = None
        self._host = None

    # GPU_Implementation6::initialize (gpu_implementation6.cpp:319-337), allocate_arrays (:385-401),
    # update_constants (:522-525)
    def initialize(self, capacity):
        self.handle = MPMHandle(self.prms, capacity, self.precision, self.device)

    def allocate_arrays(self):
        pass

    def split_hssoa_into_partitions(self):
        pass   # one partition spans the grid

    def transfer_ponts_to_device(self, soa, n=None, cohesion=None):
        self.hssoa = np.ascontiguousarray(soa, dtype=np.float64)
        self.handle.upload(self.hssoa, n, cohesion)

    def update_constants(self):
        self.handle.update_constants(self.prms)

    def reset_grid(self):
        self.handle.reset_grid()

    def p2g(self):
        self.handle.p2g()

    def receive_halos(self):
        pass   # one partition: no halo

    def update_nodes(self):
        self.handle.update_nodes(self.prms.indenter_x, self.prms.indenter_y)

    def g2p(self, recordPQ, enablePointTransfer=False):
        self.handle.g2p(recordPQ)

    def receive_points(self):
        pass   # one partition: no migration

    def record_timings(self, enablePointTransfer=False):
        pass

    def reset_indenter_force_accumulator(self):
        self.handle.reset_indenter_force_accumulator()

    def transfer_from_device(self):
        cap = max(self.handle.capacity, 1)
        if self._host is None or self._host.shape[1] < cap:
            self._host = pinned_empty((N_PTS_ARRAYS, cap))
        self.hssoa = self.handle.download(out=self._host)
        sensor, total = self.handle.sensors()
        self.indenter_sensor_total = sensor
        self.indenter_force = total
        return self.hssoa

    def evaluate_indenter_total_force(self):
        return self.indenter_force

    def synchronize(self):
        self.handle.synchronize()


class Model3D:
    """Model3D::Step for one frame of UpdateEveryNthStep substeps, driving the
    phase API exactly as the reference does (model_3d.cpp:24-112).

    capacity: host/device capacity (default: the particle count); sort: run
    RemoveDisabledAndSort (on the device) after the upload, as LoadRawPoints
    and ReadSnapshot do."""

    def __init__(self, prms, soa, cohesion=None, precision=PRECISION_FP64, device=0, capacity=None, sort=False):
        self.prms = prms.copy()
        self.gpu = GPU_Implementation6(self.prms, precision, device)
        self.gpu.initialize(soa.shape[1] if capacity is None else max(int(capacity), soa.shape[1]))
        self.gpu.transfer_ponts_to_device(soa, cohesion=cohesion)
        if sort:
            self.gpu.handle.sort()
            self.gpu.hssoa = self.gpu.handle.download()
        self.gpu.update_constants()

    @classmethod
    def from_config(cls, json_path, base_dir=None, precision=PRECISION_FP64, device=0):
        """The CLI path (cli/main.cpp:54-58): SimParams3D::ParseFile, then
        SnapshotManager::LoadRawPoints on InputRawPoints, resolved against
        base_dir (default: the working directory, as the reference does)."""
        p = SimParams3D()
        raw = ctypes.create_string_buffer(4096)
        check(LIB.mpm_params_parse_file(p, os.fspath(json_path).encode(), raw, len(raw)), "mpm_params_parse_file")
        path = raw.value.decode()
        if base_dir is not None and not os.path.isabs(path):
            path = os.path.join(base_dir, path)
        model = cls.__new__(cls)
        model.prms = p
        model.gpu = None
        SnapshotManager(model).LoadRawPoints(path, precision, device)
        return model

    @classmethod
    def from_snapshot(cls, path, partitions=0, precision=PRECISION_FP64, device=0):
        """The CLI's --resume (cli/main.cpp:44-52): SnapshotManager::ReadSnapshot."""
        model = cls.__new__(cls)
        model.prms = SimParams3D()
        model.gpu = None
        SnapshotManager(model).ReadSnapshot(path, partitions, precision, device)
        return model

    def Reset(self):
        """Model3D::Reset (model_3d.cpp:122-130)."""
        self.prms.SimulationStep = 0
        self.prms.SimulationTime = 0.0

    def Prepare(self):
        """Model3D::Prepare (model_3d.cpp:132-137)."""
        self.gpu.update_constants()

    def Step(self, substeps=None):
        p = self.prms
        simulation_time = p.SimulationTime
        count = 0
        self.gpu.reset_indenter_force_accumulator()
        n_sub = substeps if substeps is not None else None
        while True:
            simulation_time += p.InitialTimeStep
            p.indenter_x = p.indenter_x_initial + simulation_time * p.IndVelocity
            self.gpu.reset_grid()
            self.gpu.p2g()
            self.gpu.receive_halos()
            self.gpu.update_nodes()
            isZeroStep = (p.SimulationStep + count) % p.UpdateEveryNthStep == 0
            self.gpu.g2p(isZeroStep, False)
            count += 1
            if n_sub is not None and count >= n_sub:
                break
            if n_sub is None and (p.SimulationStep + count) % p.UpdateEveryNthStep == 0:
                break
        p.SimulationTime = simulation_time
        p.SimulationStep += count
        self.gpu.transfer_from_device()
        return p.SimulationTime < p.SimulationEndTime


class SnapshotManager:
    """Method-for-method mirror of the reference class (snapshotmanager.h:15-42)
    for the raw point-cloud loader, the full snapshot and resume; the files
    are the reference's (see icempm_3dm_b200.snapshot)."""

    def __init__(self, model):
        self.model = model
        self.previous_frame_exists = False

    def LoadRawPoints(self, fileName, precision=None, device=0):
        """snapshotmanager.cpp:20-113: read and place the points, allocate
        (capacity n * (1 + ExtraSpaceForIncomingPoints)), upload, sort on the
        device, Reset, Prepare."""
        m = self.model
        p, soa, capacity = _snap.load_raw_points(fileName, m.prms)
        prec = precision if precision is not None else (m.gpu.precision if m.gpu else PRECISION_FP64)
        dev = m.gpu.device if m.gpu else device
        if m.gpu is not None and m.gpu.handle is not None:
            m.gpu.handle.close()
        Model3D.__init__(m, p, soa, precision=prec, device=dev, capacity=capacity, sort=True)
        m.Reset()
        m.Prepare()
        self.previous_frame_exists = False

    def SaveSnapshot(self, outputDirectory, frame, compress=False):
        """snapshotmanager.cpp:299-340: d<frame>.h5 from the current host SoA
        (downloaded) at the handle's capacity."""
        m = self.model
        g = m.gpu
        g.transfer_from_device()
        size = g.hssoa.shape[1]
        buf = np.zeros((N_PTS_ARRAYS, g.handle.capacity), dtype=np.float64)
        buf[:, :size] = g.hssoa
        return _snap.save_snapshot(outputDirectory, frame, m.prms, buf, size, g.indenter_sensor_total, compress)

    def SaveFrame(self, outputDirectory, frame):
        """snapshotmanager.cpp:116-293: v<frame>.h5, a full frame when no
        previous frame exists, else the changed points (mpm_frame_records).
        Uses the sensors and force of the last transfer_from_device (the
        end of Model3D.Step)."""
        m = self.model
        g = m.gpu
        if g.indenter_sensor_total is None:
            g.transfer_from_device()
        prev = self.previous_frame_exists
        if not prev:
            recs = {"points": g.handle.frame_records(frame, True)}
        else:
            pv, jp, st = g.handle.frame_records(frame, False)
            recs = {"upd_pos": pv, "upd_jp": jp, "upd_status": st}
        path = _snap.save_frame(outputDirectory, frame, m.prms, g.indenter_sensor_total, g.indenter_force, prev,
                                **recs)
        self.previous_frame_exists = True
        return path

    def ReadSnapshot(self, fileName, partitions=0, precision=None, device=0):
        """snapshotmanager.cpp:346-405: parameters from the attributes, the
        points (sorted on the device when SimulationStep != 0), Prepare, and
        the indenter accumulator."""
        m = self.model
        p, hssoa, size, ind = _snap.read_snapshot(fileName, partitions)
        prec = precision if precision is not None else (m.gpu.precision if m.gpu else PRECISION_FP64)
        dev = m.gpu.device if m.gpu else device
        if m.gpu is not None and m.gpu.handle is not None:
            m.gpu.handle.close()
        Model3D.__init__(m, p, np.ascontiguousarray(hssoa[:, :size]), precision=prec, device=dev,
                         capacity=hssoa.shape[1], sort=p.SimulationStep != 0)
        m.Prepare()
        m.gpu.indenter_sensor_total = ind
        self.previous_frame_exists = False
