"""icempm_3dm_b200 — B200-native single-partition MLS-MPM step (iceMPM_3Dm hot path).

The compute path is the CUDA library libicempm_b200.so (C-ABI in
include/icempm_b200.h); this package holds its ctypes bindings, the
reference-shaped host classes and the synthetic workload generator.
"""
from ._lib import (LIB, LIB_PATH, MPMError, SimParams3D, PRECISION_FP64, PRECISION_MIXED,  # noqa: F401
                   PRECISION_FP64_SVD64, N_PTS_ARRAYS)
from .simulation import MPMHandle, GPU_Implementation6, Model3D, SnapshotManager  # noqa: F401
