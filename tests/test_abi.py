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


C_PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "icempm_b200.h"
#include "icempm_b200_testing.h"

int main(void) {
    SimParams3D p;
    char raw[256];
    int st = -1;
    mpm_params_reset(&p);
    if (mpm_params_parse_string(&p, "{\"InputRawPoints\": \"pc.h5\", \"GridX\": 64, \"GridY\": 27, "
                                    "\"GridZ\": 56, \"DomainDimensionX\": 3.3}", raw, (int)sizeof raw) != 0)
        return 2;
    if (strcmp(raw, "pc.h5") != 0 || p.GridXTotal != 64 || p.GridZ != 56) return 3;
    if (mpm_testing_sizeof_params() != sizeof(SimParams3D)) return 4;
    if (sizeof(mpm_visual_point) != 32 || sizeof(mpm_update_pos) != 28 || sizeof(mpm_update_jp) != 8 ||
        sizeof(mpm_update_status) != 8)
        return 5;
    mpm_handle* h = mpm_create(&p, MPM_PRECISION_MIXED, 1000, 0, &st);
    if (h) { mpm_destroy(h); printf("device\n"); return 0; }
    printf("status %d\n", st);
    return st == MPM_ERR_NO_DEVICE ? 0 : 6;
}
"""


def test_headers_compile_as_c_and_a_c_program_links_and_runs(tmp_path):
    """include/*.h are plain C99: a C program includes both headers, links
    against libicempm_b200.so and calls it (parameters, struct layouts,
    mpm_create, which without a GPU reports MPM_ERR_NO_DEVICE)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        return
    src = tmp_path / "abi.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "abi"
    libdir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-L", libdir, "-licempm_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.strip() in ("device", "status 103")


def test_create_rejects_grids_the_kernels_cannot_index():
    """Argument checks come before the device probe: more than 2^31 nodes,
    or (mixed precision) a grid dimension of 2047 cells or more, which the
    32-bit fixed-point positions (20 fraction bits) cannot reach."""
    p = SimParams3D()
    LIB.mpm_params_reset(p)
    st = ctypes.c_int(-1)
    p.GridXTotal, p.GridY, p.GridZ = 2100, 50, 50
    assert not LIB.mpm_create(p, 1, 100, 0, ctypes.byref(st)) and st.value == 101
    h = LIB.mpm_create(p, 0, 100, 0, ctypes.byref(st))      # FP64 takes that grid
    if h:
        LIB.mpm_destroy(h)
    assert st.value != 101
    p.GridXTotal, p.GridY, p.GridZ = 1500, 1500, 1000
    assert not LIB.mpm_create(p, 0, 100, 0, ctypes.byref(st)) and st.value == 101


def test_python_wrapper_rejects_short_host_arrays_before_the_library_reads_them():
    """Host-side size checks in MPMHandle: arrays shorter than the counts the
    library would read raise ValueError before any call crosses the ABI."""
    import numpy as np
    import pytest
    from icempm_3dm_b200 import simulation as sim

    class Fake(sim.MPMHandle):       # no device: only the checks run
        def __init__(self):
            self._h = None
            self._adj_steps = None

    h = Fake()
    soa = np.zeros((28, 10))
    with pytest.raises(ValueError):
        h.upload(np.zeros((27, 10)))
    with pytest.raises(ValueError):
        h.upload(soa, n=11)
    with pytest.raises(ValueError):
        h.upload(soa, cohesion=np.ones(9))
    with pytest.raises(sim.MPMError):
        h.adjoint_backward(np.zeros((5, 3)))
    h._adj_steps = 4
    with pytest.raises(ValueError):
        h.adjoint_backward(np.zeros((5, 3)))
