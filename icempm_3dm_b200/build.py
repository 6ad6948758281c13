"""Build recipe of the in-tree shared library libicempm_b200.so (sm_100a).

    python icempm_3dm_b200/build.py          # library only
    python icempm_3dm_b200/build.py --all    # library + CPU oracle (+ _ref)

nvcc cross-compiles for sm_100a without a GPU. The library carries the C-ABI
of include/icempm_b200.h; it has no PyTorch dependency.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libicempm_b200.so")

CU_SOURCES = ["mpm_abi.cu"]
CPP_SOURCES = ["params.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-shared",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _sources():
    return [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES]


def _deps():
    deps = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            deps.append(os.path.join(d, f))
    return deps


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build_library(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    cmd = [_nvcc()] + NVCC_FLAGS + _sources() + ["-o", OUT]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    return OUT


def build_oracle():
    """The CPU oracle (test infrastructure) and its `ref` target: the
    reference's own SVD and step kernels under oracle/_ref, built by
    oracle/Makefile from the reference tree when that tree is present (the
    Makefile names its default location; ICEMPM_REFERENCE_TREE overrides
    it)."""
    odir = os.path.join(ROOT, "oracle")
    r = subprocess.run(["make", "-C", odir], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    ref = os.environ.get("ICEMPM_REFERENCE_TREE")
    r = subprocess.run(["make", "-C", odir, "ref"] + ([f"REF={ref}"] if ref else []), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle/_ref build failed:\n" + r.stdout + r.stderr)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    if "--all" in sys.argv:
        build_oracle()
    print(OUT)
