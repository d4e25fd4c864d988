"""Test infrastructure, not the product: the checker of the POD basis.

Restates OnlinePOD::computeBasis (src/reduced_order/pod_basis_online.cpp:49-62) in numpy: the
reference state is the row mean of the snapshot matrix (:52), the snapshots are centred on it
(:59), and the basis is the thin SVD's matrix of left singular vectors (:61-62; the reference
uses Eigen's BDCSVD with ComputeThinU, LAPACK's divide-and-conquer SVD computes the same
factors here). Singular vectors are defined up to sign: `sign_rule` applies the library's rule
(the entry of largest magnitude positive) to both sides before a comparison.

Parity: the reference holds no golden POD values (no test in its tree calls OnlinePOD); this
restatement is pinned by the SVD's defining properties (tests/test_pod.py).
"""
from __future__ import annotations

import numpy as np


def compute_basis(S: np.ndarray):
    """S: ndofs x m. Returns (reference_state, singular_values, basis ndofs x m)."""
    ref = S.mean(axis=1)
    Sc = S - ref[:, None]
    U, s, _ = np.linalg.svd(Sc, full_matrices=False)
    return ref, s, U


def sign_rule(U: np.ndarray) -> np.ndarray:
    """Flip each column so that its entry of largest magnitude (the first such) is positive."""
    U = U.copy()
    for k in range(U.shape[1]):
        i = int(np.argmax(np.abs(U[:, k])))
        if U[i, k] < 0:
            U[:, k] = -U[:, k]
    return U
