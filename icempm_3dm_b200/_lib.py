"""ctypes bindings of the C-ABI library (include/icempm_b200.h).

The library is built in-tree (icempm_3dm_b200/libicempm_b200.so) by
icempm_3dm_b200/build.py. Importing this module without the library raises:
there is no CPU fallback.
"""
import ctypes
import os

from .layout import (BP00, ERR_NAMES, FE00, IDX_JP_INV, IDX_P, IDX_Q, IDX_UTILITY, N_PTS_ARRAYS,  # noqa: F401
                     POSX, PRECISION_FP64, PRECISION_FP64_SVD64, PRECISION_MIXED, STATUS_CRUSHED,
                     STATUS_DISABLED, STATUS_LIQUID, VELX, SimParams3D)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libicempm_b200.so")

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint)
_ip = ctypes.POINTER(ctypes.c_int)
_hp = ctypes.c_void_p
_pp = ctypes.POINTER(SimParams3D)

# (name, restype, argtypes) of every entry point of include/icempm_b200.h
# and include/icempm_b200_testing.h
ENTRY_POINTS = [
    ("mpm_params_reset", None, [_pp]),
    ("mpm_params_compute_lame", None, [_pp]),
    ("mpm_params_compute_camclay", None, [_pp]),
    ("mpm_params_compute_helper_variables", None, [_pp]),
    ("mpm_params_set_phi", None, [_pp, ctypes.c_double]),
    ("mpm_params_parse_file", ctypes.c_int, [_pp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
    ("mpm_params_parse_string", ctypes.c_int, [_pp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]),
    ("mpm_create", _hp, [_pp, ctypes.c_int, ctypes.c_uint, ctypes.c_int, _ip]),
    ("mpm_destroy", None, [_hp]),
    ("mpm_set_stream", ctypes.c_int, [_hp, ctypes.c_void_p]),
    ("mpm_update_constants", ctypes.c_int, [_hp, _pp]),
    ("mpm_upload_soa", ctypes.c_int, [_hp, _dp, ctypes.c_uint, ctypes.c_uint]),
    ("mpm_upload_cohesion", ctypes.c_int, [_hp, _dp, ctypes.c_uint]),
    ("mpm_download_soa", ctypes.c_int, [_hp, _dp, ctypes.c_uint, _up]),
    ("mpm_download_ids", ctypes.c_int, [_hp, _up, _up]),
    ("mpm_upload_ids", ctypes.c_int, [_hp, _up, ctypes.c_uint]),
    ("mpm_download_cohesion", ctypes.c_int, [_hp, _dp, _up]),
    ("mpm_sort", ctypes.c_int, [_hp]),
    ("mpm_set_sort_interval", ctypes.c_int, [_hp, ctypes.c_int]),
    ("mpm_set_grid_accumulation", ctypes.c_int, [_hp, ctypes.c_int]),
    ("mpm_frame_records", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _up, ctypes.c_void_p, _up,
                                         ctypes.c_void_p, _up, ctypes.c_void_p, _up]),
    ("mpm_reset_grid", ctypes.c_int, [_hp]),
    ("mpm_p2g", ctypes.c_int, [_hp]),
    ("mpm_update_nodes", ctypes.c_int, [_hp, ctypes.c_double, ctypes.c_double]),
    ("mpm_g2p", ctypes.c_int, [_hp, ctypes.c_int]),
    ("mpm_reset_indenter_force_accumulator", ctypes.c_int, [_hp]),
    ("mpm_step", ctypes.c_int, [_hp, ctypes.c_int, _dp]),
    ("mpm_sensors", ctypes.c_int, [_hp, _dp, _dp]),
    ("mpm_get_error", ctypes.c_int, [_hp]),
    ("mpm_synchronize", ctypes.c_int, [_hp]),
    ("mpm_get_params", ctypes.c_int, [_hp, _pp]),
    ("mpm_count", ctypes.c_int, [_hp, _up]),
    ("mpm_last_error_string", ctypes.c_char_p, []),
    ("mpm_host_alloc", ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    ("mpm_host_free", ctypes.c_int, [ctypes.c_void_p]),
    ("mpm_adjoint_forward", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, _dp]),
    ("mpm_adjoint_backward", ctypes.c_int, [_hp, _dp, _dp, _dp]),
    ("mpm_adjoint_state", ctypes.c_int, [_hp, _dp, ctypes.c_uint]),
    ("mpm_adjoint", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]),
    ("mpm_sort_permutation_noalloc", ctypes.c_int,
     [_pp, ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, _up, ctypes.c_void_p]),
    ("mpm_set_partition", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint]),
    ("mpm_halo_bytes", ctypes.c_size_t, [_hp]),
    ("mpm_halo_pack", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_void_p]),
    ("mpm_halo_add", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_void_p]),
    ("mpm_point_record_bytes", ctypes.c_size_t, [_hp]),
    ("mpm_points_out", ctypes.c_int, [_hp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint, _up, _up, _ip]),
    ("mpm_points_in", ctypes.c_int, [_hp, ctypes.c_void_p, ctypes.c_uint]),
    ("mpm_substep_p2g", ctypes.c_int, [_hp]),
    ("mpm_substep_update_g2p", ctypes.c_int, [_hp, ctypes.c_int, _dp]),
    ("mpm_multi_create", _hp, [_pp, ctypes.c_int, ctypes.c_uint, _ip, ctypes.c_int, _ip]),
    ("mpm_multi_destroy", None, [_hp]),
    ("mpm_multi_upload_soa", ctypes.c_int, [_hp, _dp, ctypes.c_uint, ctypes.c_uint, _dp]),
    ("mpm_multi_step", ctypes.c_int, [_hp, ctypes.c_int, _dp]),
    ("mpm_multi_download_soa", ctypes.c_int, [_hp, _dp, ctypes.c_uint, _up, _up]),
    ("mpm_multi_rebalance", ctypes.c_int, [_hp]),
    ("mpm_multi_info", ctypes.c_int, [_hp, ctypes.c_int, _ip, _ip, _up, _up]),
    ("mpm_multi_stats", ctypes.c_int, [_hp, _ip, _ip, _ip]),
    ("mpm_multi_sensors", ctypes.c_int, [_hp, _dp, _dp]),
    ("mpm_multi_reset_indenter_force_accumulator", ctypes.c_int, [_hp]),
    ("mpm_testing_svd3x3", ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]),
    ("mpm_testing_sizeof_params", ctypes.c_size_t, []),
    ("mpm_testing_step_timed", ctypes.c_int, [_hp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("mpm_testing_active_nodes", ctypes.c_int, [_hp, ctypes.POINTER(ctypes.c_longlong)]),
    ("mpm_testing_download_grid", ctypes.c_int, [_hp, _dp, ctypes.c_int]),
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `python icempm_3dm_b200/build.py` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in ENTRY_POINTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def dptr(a):
    return a.ctypes.data_as(_dp)


def uptr(a):
    return a.ctypes.data_as(_up)


class MPMError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        msg = ERR_NAMES.get(code, f"error {code}")
        if code == 100:
            msg += ": " + (LIB.mpm_last_error_string() or b"").decode(errors="replace")
        super().__init__(f"{where}: {msg} (code {code})" if where else f"{msg} (code {code})")


def check(code, where=""):
    if code != 0:
        raise MPMError(code, where)
    return code
