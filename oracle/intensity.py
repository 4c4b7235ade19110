"""ORACLE (test infrastructure): the spin-wave intensity contraction that
consumes the eigenpairs of the metric pencil, restated on the CPU.

Sunny's linear spin-wave pattern (the reference's
julia/SunnyGeneigBench/scripts/setup_sw08.jl:1-18 builds the pencil;
benchmarks/sw08_baseline.jl:99-103 reduces the eigenvectors to intensities
on an energy grid) solves Sigma u = lambda D u per q-point, with
Sigma = diag(I_m, -I_m) and D the positive-definite dynamical matrix. For
U with U^H D U = I, the Bogoliubov (para-unitary) vectors of the m
positive-energy modes are t_k = u_k / sqrt(lambda_k) with energies
omega_k = 1 / lambda_k (lambda_k > 0): t_k^H D t_k = omega_k and
t_k^H Sigma t_k = 1. The intensity of mode k is

    I_k = sum_{a,b} P_ab conj(Y_ak) Y_bk,   Y = O T,   P = I_3 - qhat qhat^T

for the caller's 3 x n one-body observable matrix O(q) (the spin-component
amplitudes of each boson: local frames, spin lengths, form factors and
phases e^{i q r} live in O) and the unit scattering direction qhat
(perpendicular projection). The spectrum on the energy grid E is
S(q, E_e) = sum_k I_k g(E_e - omega_k) with a normalised Gaussian of full
width at half maximum `fwhm`.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack


def sigma_matrix(n: int) -> np.ndarray:
    m = n // 2
    return np.diag(np.concatenate([np.ones(m), -np.ones(n - m)])).astype(np.complex128)


def gaussian(x: np.ndarray, fwhm: float) -> np.ndarray:
    sigma = fwhm / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    return np.exp(-0.5 * (x / sigma) ** 2) / (sigma * np.sqrt(2.0 * np.pi))


def sigma_intensities(D: np.ndarray, O: np.ndarray, qhat: np.ndarray, energies: np.ndarray, fwhm: float):
    """D (batch, n, n) PD dynamical matrices, O (batch, 3, n), qhat (batch, 3),
    energies (E,). Returns W (batch, n) ascending eigenvalues of the pencil
    (Sigma, D), the mode energies omega (batch, n/2) ascending, the mode
    intensities (batch, n/2) in the same order, the spectrum S (batch, E),
    and LAPACK's info per problem."""
    batch, n, _ = D.shape
    m = n // 2
    Sg = sigma_matrix(n)
    W = np.full((batch, n), np.nan)
    omega = np.full((batch, m), np.nan)
    inten = np.full((batch, m), np.nan)
    spec = np.full((batch, len(energies)), np.nan)
    info = np.zeros(batch, dtype=np.int32)
    for b in range(batch):
        w, U, inf = lapack.zhegv(Sg, D[b], itype=1, jobz="V", uplo="L")
        info[b] = inf
        if inf:
            continue
        W[b] = w
        pos = w > 0
        lam = w[pos]
        T = U[:, pos] / np.sqrt(lam)[None, :]
        om = 1.0 / lam
        Y = O[b] @ T
        P = np.eye(3) - np.outer(qhat[b], qhat[b])
        I_k = np.real(np.einsum("ak,ab,bk->k", np.conj(Y), P, Y))
        order = np.argsort(om, kind="stable")
        omega[b], inten[b] = om[order], I_k[order]
        spec[b] = (I_k[None, :] * gaussian(energies[:, None] - om[None, :], fwhm)).sum(axis=1)
    return W, omega, inten, spec, info
