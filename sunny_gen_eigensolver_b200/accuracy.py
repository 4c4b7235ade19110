"""Per-matrix accuracy measures of a generalized eigen-decomposition
H U = S U diag(W), used by the parity tests, the bench report and the serving
loop. All inputs are natural-layout numpy arrays: H, S (batch, n, n),
W (batch, n), U (batch, n, n) with U[b][:, k] the k-th eigenvector.

* `residual`      ||H U - S U diag(W)||_F / (||H||_2 ||U||_2)
* `s_orth`        max |U^H S U - I|
* `eig_err_rel`   max_k |W - W_ref| / ||H||_2   (the north-star bar)
* `eig_rel_ref`   max_k |W - W_ref| / max(|W_ref|, 1)   (the reference's own
                  acceptance metric, tests/unified/test_n54.cpp:142-147)
* `phase_err`     max_k 1 - |u_k^H S u_ref_k| over eigenvalues whose gap to
                  both neighbours is >= degen_gap (test_n54.cpp:148-162)
* `subspace_err`  for each cluster of eigenvalues closer than `cluster_tol`,
                  || (I - U_c U_c^H S) U_ref_c ||_2: distance between the two
                  S-orthonormal bases of the cluster's invariant subspace.
"""
from __future__ import annotations

import numpy as np


def _herm(X):
    return np.conj(np.swapaxes(X, -1, -2))


def norm2(M: np.ndarray) -> np.ndarray:
    return np.linalg.norm(M, ord=2, axis=(-2, -1))


def residual(H, S, W, U) -> np.ndarray:
    R = H @ U - (S @ U) * W[:, None, :]
    return np.linalg.norm(R, axis=(-2, -1)) / (norm2(H) * norm2(U))


def s_orth(S, U) -> np.ndarray:
    n = U.shape[-1]
    G = _herm(U) @ S @ U - np.eye(n)[None]
    return np.abs(G).max(axis=(-2, -1))


def eig_err_rel(H, W, W_ref) -> np.ndarray:
    return np.abs(W - W_ref).max(axis=-1) / norm2(H)


def eig_rel_ref(W, W_ref) -> np.ndarray:
    return (np.abs(W - W_ref) / np.maximum(np.abs(W_ref), 1.0)).max(axis=-1)


def phase_err(S, U, U_ref, W_ref, degen_gap: float = 1e-6) -> np.ndarray:
    out = np.zeros(U.shape[0])
    for b in range(U.shape[0]):
        inner = np.abs(np.sum(np.conj(U[b]) * (S[b] @ U_ref[b]), axis=0))
        w = W_ref[b]
        gap = np.full(w.shape, np.inf)
        gap[1:] = np.minimum(gap[1:], np.abs(np.diff(w)))
        gap[:-1] = np.minimum(gap[:-1], np.abs(np.diff(w)))
        ok = gap >= degen_gap
        out[b] = (1.0 - inner[ok]).max() if ok.any() else 0.0
    return out


def clusters(w: np.ndarray, tol: float):
    """Index ranges [lo, hi) of consecutive sorted eigenvalues closer than tol."""
    out, lo = [], 0
    for k in range(1, len(w) + 1):
        if k == len(w) or abs(w[k] - w[k - 1]) > tol:
            out.append((lo, k))
            lo = k
    return out


def subspace_err(S, U, U_ref, W_ref, cluster_tol: float) -> np.ndarray:
    out = np.zeros(U.shape[0])
    for b in range(U.shape[0]):
        worst = 0.0
        for lo, hi in clusters(W_ref[b], cluster_tol):
            Uc, Rc = U[b][:, lo:hi], U_ref[b][:, lo:hi]
            P = Rc - Uc @ (_herm(Uc) @ (S[b] @ Rc))
            worst = max(worst, np.linalg.norm(P, 2) / max(np.linalg.norm(Rc, 2), 1e-300))
        out[b] = worst
    return out
