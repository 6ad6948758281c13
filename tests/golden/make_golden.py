"""Generates the committed golden vectors of tests/golden/.

svd_ref.npz: outputs of the reference's own 3x3 SVD (simulation/helper_math.cuh,
compiled on the host from the reference tree into oracle/_ref/libref_svd.so by
`make -C oracle ref`) on seeded inputs: random matrices, near-identity
deformation gradients, rank-deficient and sign-flipped cases. The GPU box has
no reference tree; these vectors carry the reference's answers there.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as po  # noqa: E402


def svd_inputs():
    rng = np.random.default_rng(20240601)
    mats = [rng.standard_normal((400, 3, 3)),
            np.eye(3) + 1e-3 * rng.standard_normal((400, 3, 3)),
            np.eye(3) + 1e-6 * rng.standard_normal((200, 3, 3)),
            np.eye(3) + 0.05 * rng.standard_normal((200, 3, 3))]
    rd = rng.standard_normal((100, 3, 3))
    rd[:, :, 2] = 0.5 * rd[:, :, 0]                      # rank 2
    neg = np.eye(3) + 1e-3 * rng.standard_normal((100, 3, 3))
    neg[:, :, 0] *= -1                                    # det < 0
    special = np.stack([np.eye(3), np.zeros((3, 3)), np.diag([3.0, 2.0, 1.0]), np.diag([1.0, 2.0, 3.0]),
                        np.diag([1.0, 1.0, 1.0 + 1e-7]), np.ones((3, 3))])
    return np.concatenate(mats + [rd, neg, special]).reshape(-1, 9)


def main():
    if po.ref_svd_lib() is None:
        raise SystemExit("oracle/_ref/libref_svd.so is missing: run `make -C oracle ref` first")
    A = svd_inputs()
    U = np.zeros_like(A); V = np.zeros_like(A); S = np.zeros((A.shape[0], 3))
    for k in range(A.shape[0]):
        u, s, v = po.ref_svd(A[k])
        U[k] = u.reshape(9); S[k] = s; V[k] = v.reshape(9)
    np.savez_compressed(os.path.join(HERE, "svd_ref.npz"), A=A, U=U, S=S, V=V)
    print("svd_ref.npz:", A.shape[0], "matrices")


if __name__ == "__main__":
    main()
