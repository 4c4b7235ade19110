"""LAPACK-based oracles (scipy's bundled OpenBLAS/LAPACK), natural layout:
arrays of shape (batch, n, n) with M[b, i, j] = entry (i, j).

* zhegv_batch   -- LAPACK zhegv, itype=1, jobz='V', uplo='L': the ground
                   truth of the reference's tests (test_full_batched_n54.cpp
                   uses LAPACKE_zhegv; lapack_reference.cpp:186-194 zhegvd).
                   Returns W, U, info with LAPACK's info convention
                   (n + k for a non-positive-definite leading minor k of S).
* zpotrf_batch  -- stage a2 (kernel_source.hpp:244, geneig_fixed.cu:106-132).
* reduce_batch  -- stages a2-a4, C = L^-1 H L^-H as two triangular solves,
                   the order the reference's kernel uses (:244-248).
* zheev_batch   -- stage a5 on C (lower), ascending eigenvalues (:250).
* chain_batch   -- the whole reference chain restated stage by stage (:244-253),
                   U = L^-H V.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sl
from scipy.linalg import lapack


def zhegv_batch(H: np.ndarray, S: np.ndarray):
    batch, n, _ = H.shape
    W = np.full((batch, n), np.nan)
    U = np.full((batch, n, n), np.nan + 1j * np.nan)
    info = np.zeros(batch, dtype=np.int32)
    for b in range(batch):
        w, v, inf = lapack.zhegv(H[b], S[b], itype=1, jobz="V", uplo="L")
        info[b] = inf
        if inf == 0:
            W[b], U[b] = w, v
    return W, U, info


def zpotrf_batch(S: np.ndarray):
    batch, n, _ = S.shape
    L = np.zeros_like(S)
    info = np.zeros(batch, dtype=np.int32)
    for b in range(batch):
        c, inf = lapack.zpotrf(S[b], lower=1, clean=1)
        info[b] = inf
        L[b] = np.tril(c)
    return L, info


def reduce_batch(H: np.ndarray, S: np.ndarray):
    L, info = zpotrf_batch(S)
    C = np.zeros_like(H)
    for b in range(H.shape[0]):
        if info[b]:
            continue
        X = sl.solve_triangular(L[b], H[b], lower=True)                      # L^-1 H
        C[b] = sl.solve_triangular(L[b], np.conj(X.T), lower=True).conj().T  # (L^-1 (L^-1 H)^H)^H = X L^-H
    return C, L, info


def zheev_batch(C: np.ndarray):
    batch, n, _ = C.shape
    W = np.zeros((batch, n))
    V = np.zeros_like(C)
    for b in range(batch):
        w, v, inf = lapack.zheev(C[b], compute_v=1, lower=1)
        W[b], V[b] = w, v
    return W, V


def chain_batch(H: np.ndarray, S: np.ndarray):
    C, L, info = reduce_batch(H, S)
    batch, n, _ = H.shape
    W = np.full((batch, n), np.nan)
    U = np.full_like(H, np.nan)
    for b in range(batch):
        if info[b]:
            continue
        Cl = np.tril(C[b]) + np.conj(np.tril(C[b], -1).T)
        w, v = np.linalg.eigh(Cl, UPLO="L")
        W[b] = w
        U[b] = sl.solve_triangular(L[b], v, lower=True, trans="C")
    return W, U, info
