"""icempm_3dm_b200 — B200-native MLS-MPM step (iceMPM_3Dm hot path).

The compute path is the CUDA library libicempm_b200.so (C-ABI in
include/icempm_b200.h); this package holds its ctypes bindings, the
reference-shaped host classes and the synthetic workload generator.

The names below are resolved on first use: the library is loaded when a name
that needs it (LIB, MPMHandle, ...) is first taken, and loading it raises if it
is not built (there is no CPU fallback). icempm_3dm_b200.layout and
icempm_3dm_b200.generator load no library.
"""
import importlib

_EXPORTS = {
    "SimParams3D": "layout", "PRECISION_FP64": "layout", "PRECISION_MIXED": "layout",
    "PRECISION_FP64_SVD64": "layout", "N_PTS_ARRAYS": "layout",
    "LIB": "_lib", "LIB_PATH": "_lib", "MPMError": "_lib",
    "MPMHandle": "simulation", "GPU_Implementation6": "simulation", "Model3D": "simulation",
    "SnapshotManager": "simulation", "pinned_empty": "simulation",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    mod = _EXPORTS.get(name)
    if mod is None:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    value = getattr(importlib.import_module("." + mod, __name__), name)
    globals()[name] = value
    return value
