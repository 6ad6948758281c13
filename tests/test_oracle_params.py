"""The oracle's restatement of the reference's SimParams3D routines
(oracle/params.py: Reset, SetPhi, ComputeLame, ComputeCamClayParams,
ComputeHelperVariables) against the library's own (mpm_params_*), field by
field and bit for bit, on the defaults and on every synthetic workload's
parameter block. The reference arm of bench.py builds its parameter blocks
with the oracle's routines, without loading the library."""
import ctypes

import numpy as np
import pytest

from icempm_3dm_b200 import generator as gen
from icempm_3dm_b200._lib import LIB
from icempm_3dm_b200.layout import SimParams3D
from oracle import params as oracle_params


def fields_equal(a, b):
    diff = []
    for name, _ in SimParams3D._fields_:
        va, vb = getattr(a, name), getattr(b, name)
        if name == "BlockCutout":
            va, vb = list(va), list(vb)
        if np.asarray(va, dtype=np.float64).tobytes() != np.asarray(vb, dtype=np.float64).tobytes():
            diff.append((name, va, vb))
    return diff


def test_reset_equals_the_librarys():
    a, b = SimParams3D(), SimParams3D()
    oracle_params.reset(a)
    LIB.mpm_params_reset(b)
    assert fields_equal(a, b) == []
    assert bytes(a) == bytes(b)


@pytest.mark.parametrize("name", sorted(gen.CONFIGS))
def test_workload_parameter_blocks_equal_the_librarys(name):
    cfg = gen.CONFIGS[name]
    a = gen.make_params(cfg, ops=oracle_params.OPS)
    b = gen.make_params(cfg)
    assert fields_equal(a, b) == []


def test_helper_variables_with_partitions_and_odd_sizes():
    for parts, npts, frac in ((1, 250_000, 0.05), (3, 1_000_001, 0.07), (8, 7, 0.5)):
        a, b = SimParams3D(), SimParams3D()
        for p in (a, b):
            ctypes.memset(ctypes.byref(p), 0, ctypes.sizeof(p))
        oracle_params.reset(a)
        LIB.mpm_params_reset(b)
        for p in (a, b):
            p.nPartitions, p.nPtsTotal, p.PointsTransferBufferFraction = parts, npts, frac
            p.InitialTimeStep, p.GridXTotal, p.DomainDimensionX = 7.3e-6, 333, 2.71
        oracle_params.compute_helper_variables(a)
        LIB.mpm_params_compute_helper_variables(b)
        assert fields_equal(a, b) == []
