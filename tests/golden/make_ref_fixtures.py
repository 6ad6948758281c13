"""Generates tests/golden/ref_steps.npz: runs of the reference's own step
kernels on seeded inputs, for the GPU parity tests.

The kernels are simulation/mpm_kernels.cuh of the reference, compiled
unmodified as host C++ into oracle/_ref/libref_mpm.so by `make -C oracle ref`
(oracle/ref_kernels.cpp, Eigen-API stand-in in oracle/refshim/), driven
serially in index order by oracle.pyoracle.RefSim as GPU_Implementation6
drives one partition. The GPU box has no reference tree; these arrays carry
the reference's answers there.

Per case <c>: <c>_params (the SimParams3D bytes, the reference's layout),
<c>_soa (28 x n input), <c>_hist (force history [steps, 3]), <c>_out (28 x n
state after the run). Cases:
  crushed   elastic, crushed (compression and tension, Jp_inv < 1) and
            strongly strained particles under the indenter
  liquid    20 % liquid particles at the water tank's stiffness (E = 1e8)
            and per-grain strength variability 0.5 with grain ids 0..999
  halo      GridHaloSize 4 and the indenter in contact from the first substep

    make -C oracle ref && python tests/golden/make_ref_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from icempm_3dm_b200 import generator as gen  # noqa: E402
from icempm_3dm_b200.layout import IDX_UTILITY  # noqa: E402
from oracle import params as oracle_params  # noqa: E402
from oracle import pyoracle as po  # noqa: E402
from tests.helpers import perturbed_block, util_as_double, util_bits  # noqa: E402

STEPS = 20
N = 600


def fixture_cases():
    ops = oracle_params.OPS
    out = {}
    prms, soa = perturbed_block(n=N, seed=21, dims=(0.1, 0.06, 0.06), ops=ops)
    out["crushed"] = (prms, soa)
    prms, soa = perturbed_block(n=N, seed=22, liquid_frac=0.2, youngs=1e8, dims=(0.1, 0.06, 0.06), ops=ops)
    prms.GrainVariability = 0.5
    bits = util_bits(soa).copy()
    bits |= np.random.default_rng(22).integers(0, 1000, soa.shape[1])
    soa[IDX_UTILITY] = util_as_double(bits)
    out["liquid"] = (prms, soa)
    prms, soa, _ = gen.small_block(n=N, seed=23, dims=(0.1, 0.06, 0.06), halo=4, ops=ops)
    rng = np.random.default_rng(23)
    soa[7:10] = 0.1 * rng.standard_normal((3, soa.shape[1]))
    soa[10:19] += 1e-3 * rng.standard_normal((9, soa.shape[1]))
    prms.indenter_x_initial += 2 * prms.cellsize
    prms.indenter_x = prms.indenter_x_initial
    out["halo"] = (prms, soa)
    return out


def main():
    if po.ref_mpm_lib() is None:
        raise SystemExit("oracle/_ref/libref_mpm.so is missing: run `make -C oracle ref` first")
    arrays = {"steps": np.array(STEPS)}
    for name, (prms, soa) in fixture_cases().items():
        n = soa.shape[1]
        sim = po.RefSim(prms, soa, n)
        hist, err = sim.step(STEPS)
        if err:
            raise SystemExit(f"case {name}: reference error byte {err}")
        arrays[f"{name}_params"] = np.frombuffer(bytes(prms), dtype=np.uint8)
        arrays[f"{name}_soa"] = np.ascontiguousarray(soa)
        arrays[f"{name}_hist"] = hist
        arrays[f"{name}_out"] = sim.soa
        crushed = int(((util_bits(sim.soa) & 0x10000) != 0).sum())
        print(f"{name}: {n} particles, {STEPS} substeps, |force| max {np.abs(hist).max():.4g} N, "
              f"{crushed} crushed")
    path = os.path.join(HERE, "ref_steps.npz")
    np.savez_compressed(path, **arrays)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
