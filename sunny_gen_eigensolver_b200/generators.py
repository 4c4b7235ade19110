"""Seeded synthetic (H, S) batches with the shapes and value distributions of
the workloads this solver is measured on (the reference's Sunny.jl SW08
dispersion problems are not reproducible here, so these stand in for them).

Baseline pair at size n = 2m, complex128:
  H = [[A, B], [conj(B), conj(A)]] with A = (G + G^H)/2, B = (G' + G'^T)/2,
      G, G' complex N(0,1) (real and imaginary parts each N(0,1)), shifted by
      c I so that lambda_min(H) = 0.1 ||H||_2 (the BdG block structure of a
      spin-wave dynamical matrix, positive definite);
  S = Q diag(d) Q^H, Q Haar-random unitary (QR of a complex Gaussian with the
      phases of R's diagonal folded into Q), d log-uniform on [1, kappa].
Sunny call pattern (`run_kernel!(solver, Sigma, H_dyn)` in the reference's
setup_sw08.jl:16-18, compare_pr8.jl:49-53): H = Sigma = diag(I_m, -I_m), the
indefinite metric, and S = the positive-definite BdG matrix above.

Everything is generated in natural layout: arrays of shape (batch, n, n)
with M[b, i, j] = entry (i, j).
"""
from __future__ import annotations

import numpy as np

DEFAULT_KAPPA = 100.0


def _hermitian_bdg_np(rng: np.random.Generator, n: int, batch: int) -> np.ndarray:
    if n % 2:
        raise ValueError("BdG-structured H needs even n")
    m = n // 2
    G = rng.standard_normal((batch, m, m)) + 1j * rng.standard_normal((batch, m, m))
    A = 0.5 * (G + np.conj(np.swapaxes(G, -1, -2)))
    G2 = rng.standard_normal((batch, m, m)) + 1j * rng.standard_normal((batch, m, m))
    Bm = 0.5 * (G2 + np.swapaxes(G2, -1, -2))
    H = np.empty((batch, n, n), dtype=np.complex128)
    H[:, :m, :m] = A
    H[:, :m, m:] = Bm
    H[:, m:, :m] = np.conj(Bm)
    H[:, m:, m:] = np.conj(A)
    ev = np.linalg.eigvalsh(H)
    lo, hi = ev[:, 0], ev[:, -1]
    c = (0.1 * hi - lo) / 0.9
    H += c[:, None, None] * np.eye(n)[None]
    return H


def _spd_haar_np(rng: np.random.Generator, n: int, batch: int, kappa: float) -> np.ndarray:
    X = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
    Q, R = np.linalg.qr(X)
    ph = np.diagonal(R, axis1=-2, axis2=-1)
    ph = ph / np.abs(ph)
    Q = Q * ph[:, None, :]
    d = np.exp(rng.uniform(0.0, np.log(kappa), size=(batch, n)))
    S = (Q * d[:, None, :]) @ np.conj(np.swapaxes(Q, -1, -2))
    return 0.5 * (S + np.conj(np.swapaxes(S, -1, -2)))


def baseline_problems(n: int, batch: int, seed: int, kappa: float = DEFAULT_KAPPA):
    """(H, S) natural-layout numpy batches of the baseline distribution."""
    rng = np.random.Generator(np.random.PCG64(seed))
    H = _hermitian_bdg_np(rng, n, batch)
    S = _spd_haar_np(rng, n, batch, kappa)
    return H, S


def spawned_problems(n: int, batch: int, seed: int, kappa: float = DEFAULT_KAPPA):
    """Baseline distribution with one independent substream per problem:
    problem b is drawn from PCG64(SeedSequence(seed).spawn(batch)[b]), so any
    problem regenerates on its own. The parity set of 256 problems at N=54 is
    spawned_problems(54, 256, 20261203)."""
    H = np.empty((batch, n, n), dtype=np.complex128)
    S = np.empty((batch, n, n), dtype=np.complex128)
    for b, ss in enumerate(np.random.SeedSequence(seed).spawn(batch)):
        rng = np.random.Generator(np.random.PCG64(ss))
        H[b] = _hermitian_bdg_np(rng, n, 1)[0]
        S[b] = _spd_haar_np(rng, n, 1, kappa)[0]
    return H, S


def sigma_metric_problems(n: int, batch: int, seed: int):
    """Sunny call pattern: H = diag(I_m, -I_m) (indefinite), S = PD BdG matrix."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = n // 2
    S = _hermitian_bdg_np(rng, n, batch)
    sig = np.concatenate([np.ones(m), -np.ones(n - m)])
    H = np.broadcast_to(np.diag(sig).astype(np.complex128), (batch, n, n)).copy()
    return H, S


def baseline_problems_torch(n: int, batch: int, seed: int, kappa: float = DEFAULT_KAPPA,
                            device="cuda", chunk: int = 8192):
    """Same distribution generated on the GPU with torch (input preparation for
    large benchmark batches only; torch.linalg here is not the solver)."""
    import torch
    if n % 2:
        raise ValueError("BdG-structured H needs even n")
    m = n // 2
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    H = torch.empty((batch, n, n), dtype=torch.complex128, device=device)
    S = torch.empty((batch, n, n), dtype=torch.complex128, device=device)
    eye = torch.eye(n, dtype=torch.complex128, device=device)
    for off in range(0, batch, chunk):
        b = min(chunk, batch - off)
        def cn(*shape):
            re = torch.randn(*shape, generator=gen, dtype=torch.float64, device=device)
            im = torch.randn(*shape, generator=gen, dtype=torch.float64, device=device)
            return torch.complex(re, im)
        G = cn(b, m, m)
        A = 0.5 * (G + G.conj().transpose(-1, -2))
        G2 = cn(b, m, m)
        Bm = 0.5 * (G2 + G2.transpose(-1, -2))
        Hc = torch.cat([torch.cat([A, Bm], dim=2), torch.cat([Bm.conj(), A.conj()], dim=2)], dim=1)
        ev = torch.linalg.eigvalsh(Hc)
        c = (0.1 * ev[:, -1] - ev[:, 0]) / 0.9
        Hc = Hc + c[:, None, None].to(torch.complex128) * eye
        H[off:off + b] = Hc
        X = cn(b, n, n)
        Q, R = torch.linalg.qr(X)
        ph = torch.diagonal(R, dim1=-2, dim2=-1)
        ph = ph / ph.abs()
        Q = Q * ph[:, None, :]
        u = torch.rand((b, n), generator=gen, dtype=torch.float64, device=device)
        d = torch.exp(u * np.log(kappa)).to(torch.complex128)
        Sc = (Q * d[:, None, :]) @ Q.conj().transpose(-1, -2)
        S[off:off + b] = 0.5 * (Sc + Sc.conj().transpose(-1, -2))
    return H, S
