"""Pins the oracle's 3x3 SVD to the reference's own (helper_math.cuh):
bit-exact against the committed golden vectors generated from the reference
compiled on the host, and against oracle/_ref when it is built."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "svd_ref.npz")


def test_oracle_svd_bit_exact_on_reference_golden_vectors():
    g = np.load(GOLDEN)
    for k in range(g["A"].shape[0]):
        u, s, v = po.svd(g["A"][k])
        assert np.array_equal(u.reshape(9), g["U"][k]), k
        assert np.array_equal(s, g["S"][k]), k
        assert np.array_equal(v.reshape(9), g["V"][k]), k


def test_oracle_svd_bit_exact_against_compiled_reference():
    if po.ref_svd_lib() is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(123)
    for k in range(3000):
        A = rng.standard_normal((3, 3)) if k % 2 else np.eye(3) + 1e-4 * rng.standard_normal((3, 3))
        u1, s1, v1 = po.svd(A)
        u2, s2, v2 = po.ref_svd(A)
        assert np.array_equal(u1, u2) and np.array_equal(s1, s2) and np.array_equal(v1, v2), k


def test_svd_constants_are_the_reference_floats():
    import struct
    # helper_math.cuh:10-16 bit patterns; cos(pi/8) is one ulp above rounding
    for bits, val in ((1053028117, float.fromhex("0x1.87de2ap-2")), (1064076127, float.fromhex("0x1.d906bep-1")),
                      (1085964922, float.fromhex("0x1.7504f4p+2"))):
        assert struct.unpack("<f", struct.pack("<I", bits))[0] == val


def test_f64_variant_is_accurate():
    rng = np.random.default_rng(5)
    for k in range(500):
        A = rng.standard_normal((3, 3)) if k % 2 else np.eye(3) + 1e-4 * rng.standard_normal((3, 3))
        u, s, v = po.svd(A, "f64", 8)
        assert np.abs(u @ np.diag(s) @ v.T - A).max() < 1e-13 * max(1.0, np.abs(A).max())
        assert np.abs(u.T @ u - np.eye(3)).max() < 1e-13
        assert np.allclose(np.sort(np.abs(s)), np.sort(np.linalg.svd(A, compute_uv=False)), rtol=1e-12, atol=1e-14)
