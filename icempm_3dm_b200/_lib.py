"""ctypes bindings of the C-ABI library (include/icempm_b200.h).

The library is built in-tree (icempm_3dm_b200/libicempm_b200.so) by
icempm_3dm_b200/build.py. Importing this module without the library raises:
there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libicempm_b200.so")

# Row indices of the particle SoA (parameters_sim_3d.h:29-38).
IDX_UTILITY, IDX_P, IDX_Q, IDX_JP_INV = 0, 1, 2, 3
POSX, VELX, FE00, BP00 = 4, 7, 10, 19
N_PTS_ARRAYS = 28

STATUS_CRUSHED = 0x10000
STATUS_DISABLED = 0x20000
STATUS_LIQUID = 0x40000

PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRECISION_FP64_SVD64 = 2

ERR_NAMES = {
    0: "ok", 5: "receive overflow",
    70: "particle outside grid (-x)", 71: "particle outside grid (-y)", 72: "particle outside grid (-z)",
    73: "particle outside grid (+x)", 74: "particle outside grid (+y)", 75: "particle outside grid (+z)",
    100: "CUDA runtime error", 101: "invalid argument", 102: "capacity exceeded", 103: "no suitable CUDA device",
    104: "configuration file not found", 105: "configuration file is not JSON / wrong key type",
    106: "config parameter missing (InputRawPoints)", 107: "cell key outside the grid",
    108: "call out of order", 109: "size beyond the fixed scratch of the allocation-free sort",
    110: "a bounded wait on an asynchronous copy in a kernel ran out",
}


class SimParams3D(ctypes.Structure):
    """Same field order and C types as the reference's SimParams3D
    (simulation/parameters_sim_3d.h:40-90) and include/sim_params_3d.h."""
    _fields_ = [
        ("SetupType", ctypes.c_int),
        ("nPtsTotal", ctypes.c_int),
        ("GridXTotal", ctypes.c_int), ("GridY", ctypes.c_int), ("GridZ", ctypes.c_int),
        ("IndenterSubdivisions", ctypes.c_int),
        ("DomainDimensionX", ctypes.c_double),
        ("InitialTimeStep", ctypes.c_double), ("SimulationEndTime", ctypes.c_double),
        ("SimulationTime", ctypes.c_double),
        ("UpdateEveryNthStep", ctypes.c_int),
        ("SnapshotPeriod", ctypes.c_int),
        ("SimulationStep", ctypes.c_int),
        ("Gravity", ctypes.c_double), ("Density", ctypes.c_double), ("WaterDensity", ctypes.c_double),
        ("PoissonsRatio", ctypes.c_double), ("YoungsModulus", ctypes.c_double),
        ("DragGlobal", ctypes.c_double),
        ("lambda_", ctypes.c_double), ("mu", ctypes.c_double), ("kappa", ctypes.c_double),
        ("IceCompressiveStrength", ctypes.c_double), ("IceTensileStrength", ctypes.c_double),
        ("IceShearStrength", ctypes.c_double), ("IceTensileStrength2", ctypes.c_double),
        ("NACC_beta", ctypes.c_double),
        ("DP_tan_phi", ctypes.c_double), ("DP_threshold_p", ctypes.c_double),
        ("GrainVariability", ctypes.c_double),
        ("IndDiameter", ctypes.c_double), ("IndRSq", ctypes.c_double), ("IndVelocity", ctypes.c_double),
        ("IndDepth", ctypes.c_double),
        ("cellsize", ctypes.c_double),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double),
        ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("BlockCutout", ctypes.c_double * 3),
        ("ParticleVolume", ctypes.c_double), ("ParticleMass", ctypes.c_double),
        ("ParticleViewSize", ctypes.c_double), ("LiquidParticleMass", ctypes.c_double),
        ("indenter_x", ctypes.c_double), ("indenter_x_initial", ctypes.c_double),
        ("indenter_y", ctypes.c_double), ("indenter_y_initial", ctypes.c_double),
        ("Volume", ctypes.c_double),
        ("nPartitions", ctypes.c_int),
        ("GridHaloSize", ctypes.c_int),
        ("PointTransferFrequency", ctypes.c_int),
        ("VectorCapacity_transfer", ctypes.c_int),
        ("ExtraSpaceForIncomingPoints", ctypes.c_double),
        ("PointsTransferBufferFraction", ctypes.c_double),
        ("RebalanceThresholdFreeSpaceRemaining", ctypes.c_double),
        ("RebalanceThresholdDisabledPercentage", ctypes.c_double),
        ("dt_vol_Dpinv", ctypes.c_double), ("dt_Gravity", ctypes.c_double), ("vmax", ctypes.c_double),
        ("vmax_squared", ctypes.c_double),
        ("gbOffset", ctypes.c_int),
        ("cellsize_inv", ctypes.c_double), ("Dp_inv", ctypes.c_double),
        ("tpb_P2G", ctypes.c_int), ("tpb_Upd", ctypes.c_int), ("tpb_G2P", ctypes.c_int),
        ("animation_threshold_pos", ctypes.c_double),
    ]

    def copy(self):
        c = SimParams3D()
        ctypes.pointer(c)[0] = self
        return c


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
    ("mpm_sort", ctypes.c_int, [_hp]),
    ("mpm_set_sort_interval", ctypes.c_int, [_hp, ctypes.c_int]),
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
    ("mpm_adjoint_forward", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, _dp]),
    ("mpm_adjoint_backward", ctypes.c_int, [_hp, _dp, _dp, _dp]),
    ("mpm_adjoint_state", ctypes.c_int, [_hp, _dp, ctypes.c_uint]),
    ("mpm_adjoint", ctypes.c_int, [_hp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]),
    ("mpm_sort_permutation_noalloc", ctypes.c_int,
     [_pp, ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p, _up, ctypes.c_void_p]),
    ("mpm_testing_set_p2g_variant", ctypes.c_int, [_hp, ctypes.c_int]),
    ("mpm_testing_set_g2p_variant", ctypes.c_int, [_hp, ctypes.c_int]),
    ("mpm_testing_svd3x3", ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int]),
    ("mpm_testing_sizeof_params", ctypes.c_size_t, []),
    ("mpm_testing_step_timed", ctypes.c_int, [_hp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("mpm_testing_active_nodes", ctypes.c_int, [_hp, ctypes.POINTER(ctypes.c_longlong)]),
    ("mpm_testing_copy_wait_timeout", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
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
