"""CPU ORACLE — test infrastructure, not product code.

ctypes bindings of oracle/liboracle.so (the C++ restatement of the
reference step, see mpm_oracle.h), of oracle/_ref/libref_svd.so (the
reference's own helper_math.cuh SVD compiled on the host) and of
oracle/_ref/libref_mpm.so (the reference's own mpm_kernels.cuh compiled on
the host, driven by RefSim). Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg and reference arm import this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _load():
    path = os.path.join(_HERE, "liboracle.so")
    if not os.path.exists(path):
        raise RuntimeError("oracle/liboracle.so is not built: run `make -C oracle`")
    lib = ctypes.CDLL(path)
    lib.or_grid_nodes.restype = ctypes.c_longlong
    lib.or_grid_nodes.argtypes = [ctypes.c_void_p]
    lib.or_svd3x3_f32.argtypes = [_dp, _dp, _dp, _dp]
    lib.or_svd3x3_f64.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int]
    lib.or_cell_key.restype = ctypes.c_int
    lib.or_cell_key.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.or_sort_permutation.restype = ctypes.c_uint
    lib.or_sort_permutation.argtypes = [ctypes.c_void_p, _dp, ctypes.c_uint, ctypes.c_uint, _up]
    lib.or_p2g.restype = ctypes.c_int
    lib.or_p2g.argtypes = [ctypes.c_void_p, _dp, ctypes.c_uint, ctypes.c_uint, _dp, ctypes.c_int]
    lib.or_update_nodes.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, ctypes.c_int]
    lib.or_g2p.restype = ctypes.c_int
    lib.or_g2p.argtypes = [ctypes.c_void_p, _dp, ctypes.c_uint, ctypes.c_uint, _dp, ctypes.c_int, _dp,
                           ctypes.c_int, ctypes.c_int]
    lib.or_step.restype = ctypes.c_int
    lib.or_step.argtypes = [ctypes.c_void_p, _dp, ctypes.c_uint, ctypes.c_uint, _dp, _dp, _dp, _dp,
                            ctypes.c_int, ctypes.c_int]
    lib.or_svd3x3_dual.argtypes = [_dp] * 8 + [ctypes.c_int]
    lib.or_dual_steps.restype = ctypes.c_int
    lib.or_dual_steps.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_uint, ctypes.c_uint, _dp, _dp,
                                  ctypes.c_double, ctypes.c_int, _dp, _dp]
    return lib


LIB = _load()


def ref_svd_lib():
    """The reference's own SVD compiled on the host, or None if not built."""
    path = os.path.join(_HERE, "_ref", "libref_svd.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    lib.ref_svd3x3.argtypes = [_dp, _dp, _dp, _dp]
    return lib


def svd(a, mode="f32", sweeps=8):
    """3x3 SVD of the oracle: mode f32 = reference semantics, f64 = double."""
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    u = np.zeros(9); s = np.zeros(3); v = np.zeros(9)
    if mode == "f32":
        LIB.or_svd3x3_f32(_ptr(a), _ptr(u), _ptr(s), _ptr(v))
    else:
        LIB.or_svd3x3_f64(_ptr(a), _ptr(u), _ptr(s), _ptr(v), sweeps)
    return u.reshape(3, 3), s, v.reshape(3, 3)


def svd_dual(a, da, sweeps=8):
    """Forward-mode derivative of the FP64 SVD along da: ((U, S, V), (dU, dS, dV))."""
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    da = np.ascontiguousarray(da, dtype=np.float64).reshape(9)
    out = [np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(3), np.zeros(9), np.zeros(9)]
    LIB.or_svd3x3_dual(_ptr(a), _ptr(da), *[_ptr(o) for o in out], sweeps)
    u, du, s, ds, v, dv = out
    return (u.reshape(3, 3), s, v.reshape(3, 3)), (du.reshape(3, 3), ds, dv.reshape(3, 3))


def dual_steps(prms, soa, nsteps, dsoa=None, p0=None, dp0=None, dE=0.0):
    """FP64 dual-number forward-mode derivative of nsteps substeps (FP64 SVD).

    Returns (force_hist, dforce_hist, soa_final, dsoa_final); the tangents are
    the directional derivatives along (dsoa, dp0, dE). prms is not modified.
    """
    import copy
    P = copy.copy(prms)
    s = np.array(soa, dtype=np.float64, copy=True, order="C")
    ds = np.zeros_like(s) if dsoa is None else np.array(dsoa, dtype=np.float64, copy=True, order="C")
    n = s.shape[1]
    hist = np.zeros((nsteps, 3))
    dhist = np.zeros((nsteps, 3))
    p0p = None
    if p0 is not None:
        p0 = np.ascontiguousarray(p0, dtype=np.float64)
        p0p = _ptr(p0)
    if dp0 is not None:
        dp0 = np.ascontiguousarray(dp0, dtype=np.float64)
    err = LIB.or_dual_steps(ctypes.byref(P), _ptr(s), _ptr(ds), n, n, p0p,
                            _ptr(dp0) if dp0 is not None else None, dE, nsteps, _ptr(hist), _ptr(dhist))
    if err:
        raise RuntimeError(f"oracle dual step error {err}")
    return hist, dhist, s, ds


def ref_svd(a):
    lib = ref_svd_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/libref_svd.so is not built")
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    u = np.zeros(9); s = np.zeros(3); v = np.zeros(9)
    lib.ref_svd3x3(_ptr(a), _ptr(u), _ptr(s), _ptr(v))
    return u.reshape(3, 3), s, v.reshape(3, 3)


def grid_nodes(prms):
    return int(LIB.or_grid_nodes(ctypes.byref(prms)))


def cell_key(prms, x, y, z):
    return LIB.or_cell_key(ctypes.byref(prms), x, y, z)


def sort_permutation(prms, soa, n):
    """Stable RemoveDisabledAndSort permutation over the first n particles."""
    soa = np.ascontiguousarray(soa, dtype=np.float64)
    pitch = soa.shape[1]
    perm = np.zeros(n, dtype=np.uint32)
    m = LIB.or_sort_permutation(ctypes.byref(prms), _ptr(soa), pitch, n, _ptr(perm, _up))
    return perm[:m]


def p2g(prms, soa, n, nthreads=1):
    grid = np.zeros((4, grid_nodes(prms)))
    pitch = soa.shape[1]
    err = LIB.or_p2g(ctypes.byref(prms), _ptr(soa), pitch, n, _ptr(grid), nthreads)
    return grid, err


def update_nodes(prms, grid, ind_x, ind_y, sensor=None, nthreads=1):
    f = np.zeros(3)
    if sensor is None:
        sensor = np.zeros(3 * prms.IndenterSubdivisions * prms.GridZ)
    LIB.or_update_nodes(ctypes.byref(prms), _ptr(grid), ind_x, ind_y, _ptr(sensor), _ptr(f), nthreads)
    return f, sensor


def g2p(prms, soa, n, grid, record_pq=False, p0=None, svd_mode=0, nthreads=1):
    p0p = _ptr(p0) if p0 is not None else None
    return LIB.or_g2p(ctypes.byref(prms), _ptr(soa), soa.shape[1], n, _ptr(grid), int(record_pq), p0p,
                      svd_mode, nthreads)


class OracleSim:
    """Runs substeps of Model3D::Step on a private copy of the SoA."""

    def __init__(self, prms, soa, n, p0=None, svd_mode=0, nthreads=1):
        import copy
        self.prms = copy.copy(prms)
        self.soa = np.array(soa, dtype=np.float64, copy=True, order="C")
        self.n = n
        self.p0 = None if p0 is None else np.ascontiguousarray(p0, dtype=np.float64)
        self.svd_mode = svd_mode
        self.nthreads = nthreads
        self.grid = np.zeros((4, grid_nodes(self.prms)))
        self.sensor = np.zeros(3 * self.prms.IndenterSubdivisions * self.prms.GridZ)

    def step(self, nsteps=1):
        hist = np.zeros((nsteps, 3))
        err = 0
        f = np.zeros(3)
        p0p = _ptr(self.p0) if self.p0 is not None else None
        for s in range(nsteps):
            e = LIB.or_step(ctypes.byref(self.prms), _ptr(self.soa), self.soa.shape[1], self.n, _ptr(self.grid),
                            _ptr(self.sensor), _ptr(f), p0p, self.svd_mode, self.nthreads)
            hist[s] = f
            if e and not err:
                err = e
        return hist, err


# ------------------------------------------------------------------------
# The reference's own step kernels (oracle/_ref/libref_mpm.so: mpm_kernels.cuh
# compiled as host C++ from the reference tree, see oracle/ref_kernels.cpp)

_ip = ctypes.POINTER(ctypes.c_int)


def ref_mpm_lib():
    """The reference's own kernels compiled on the host, or None if not built."""
    path = os.path.join(_HERE, "_ref", "libref_mpm.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    lib.ref_sizeof_params.restype = ctypes.c_size_t
    lib.ref_params_layout.argtypes = [ctypes.POINTER(ctypes.c_size_t)]
    lib.ref_set_params.restype = ctypes.c_int
    lib.ref_set_params.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    lib.ref_error.restype = ctypes.c_int
    lib.ref_p2g.argtypes = [ctypes.c_int] * 5 + [_dp, _dp, ctypes.c_int]
    lib.ref_receive_halos.argtypes = [ctypes.c_int] * 3 + [_dp, _dp, _dp]
    lib.ref_update_nodes.argtypes = [ctypes.c_double, ctypes.c_double] + [ctypes.c_int] * 3 + [_dp, _dp,
                                                                                                  ctypes.c_int]
    lib.ref_g2p.argtypes = [ctypes.c_int] * 7 + [_dp, _dp, _ip, ctypes.c_int, _dp, _dp, ctypes.c_int]
    lib.ref_receive_points.argtypes = [ctypes.c_int] * 3 + [_dp, _dp]
    return lib


def reference_tree():
    """The reference source tree oracle/_ref was built from (its Makefile
    records the path), or None when that tree is not on this machine."""
    try:
        with open(os.path.join(_HERE, "_ref", "reference_tree")) as f:
            path = f.read().strip()
    except OSError:
        return None
    return path if os.path.isdir(os.path.join(path, "simulation")) else None


class RefSim:
    """Substeps of Model3D::Step (model_3d.cpp:35-51) for one partition,
    driven as GPU_Implementation6 drives its partition (reset_grid, p2g,
    update_nodes, g2p; gpu_implementation6.cpp:18-133,
    gpu_partition_3d.cu:222-292), through the reference's own kernels.

    nthreads <= 1 runs each kernel serially in index order (deterministic);
    more runs it over OpenMP threads. The grid is one partition's buffer of
    4 arrays of (GridXTotal + 2 GridHaloSize) GridY GridZ doubles (the
    halo-transfer slabs of gpu_partition_3d.cu:88-95 are not needed with one
    partition). force of a substep = the sum of that substep's sensor bins.
    """

    def __init__(self, prms, soa, n, nthreads=1):
        import copy
        lib = ref_mpm_lib()
        if lib is None:
            raise RuntimeError("oracle/_ref/libref_mpm.so is not built (make -C oracle ref)")
        self.lib = lib
        self.prms = copy.copy(prms)
        self.soa = np.array(soa, dtype=np.float64, copy=True, order="C")
        self.n = n
        self.nthreads = nthreads
        P = self.prms
        self.nodes = (P.GridXTotal + 2 * P.GridHaloSize) * P.GridY * P.GridZ
        self.grid = np.zeros((4, self.nodes))
        self.sensor = np.zeros(3 * P.IndenterSubdivisions * P.GridZ)
        self.step_sensor = np.zeros_like(self.sensor)
        cap = max(int(P.VectorCapacity_transfer), 1)
        self.cap = cap
        self.xfer = [np.zeros(cap * 28), np.zeros(cap * 28)]
        self.utility = np.zeros(3, dtype=np.int32)
        self.count_unupdated = 0

    def _upload_params(self):
        if self.lib.ref_set_params(ctypes.byref(self.prms), ctypes.sizeof(self.prms)) != 0:
            raise RuntimeError("SimParams3D layout differs from the reference's")

    def p2g(self):
        P = self.prms
        self.lib.ref_p2g(P.GridXTotal, 0, self.nodes, self.n, self.soa.shape[1], _ptr(self.soa), _ptr(self.grid),
                         self.nthreads)

    def update_nodes(self, ind_x, ind_y):
        self.step_sensor[:] = 0
        self.lib.ref_update_nodes(ind_x, ind_y, self.nodes, 0, self.nodes, _ptr(self.grid),
                                  _ptr(self.step_sensor), self.nthreads)
        self.sensor += self.step_sensor
        return self.step_sensor.reshape(-1, 3).sum(axis=0)

    def g2p(self, record_pq, enable_transfer=False):
        P = self.prms
        self.utility[:] = 0
        self.lib.ref_g2p(int(record_pq), int(enable_transfer), P.GridXTotal, 0, self.nodes, self.n,
                         self.soa.shape[1], _ptr(self.soa), _ptr(self.grid), _ptr(self.utility, _ip), self.cap,
                         _ptr(self.xfer[0]), _ptr(self.xfer[1]), self.nthreads)

    def step(self, nsteps=1):
        """nsteps substeps; returns (force history [nsteps, 3], error byte)."""
        P = self.prms
        self._upload_params()
        hist = np.zeros((nsteps, 3))
        t = P.SimulationTime
        for s in range(nsteps):
            t += P.InitialTimeStep
            P.indenter_x = P.indenter_x_initial + t * P.IndVelocity
            self.grid[:] = 0
            self.p2g()
            hist[s] = self.update_nodes(P.indenter_x, P.indenter_y)
            is_zero = (P.SimulationStep + s) % P.UpdateEveryNthStep == 0
            self.g2p(is_zero)
        P.SimulationTime = t
        P.SimulationStep += nsteps
        return hist, self.lib.ref_error()
