"""The C-ABI library loads and exports every entry point that include/*.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from icempm_3dm_b200 import _lib
from icempm_3dm_b200._lib import LIB, SimParams3D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("icempm_b200.h", "icempm_b200_testing.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mpm_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(LIB, n), n


def test_bindings_cover_the_headers():
    bound = {name for name, _, _ in _lib.ENTRY_POINTS}
    assert declared_functions() <= bound


def test_params_struct_layout_matches_library():
    assert ctypes.sizeof(SimParams3D) == LIB.mpm_testing_sizeof_params()


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    p = SimParams3D()
    LIB.mpm_params_reset(p)
    st = ctypes.c_int(-1)
    h = LIB.mpm_create(p, 0, 100, 0, ctypes.byref(st))
    assert not h and st.value == 103
