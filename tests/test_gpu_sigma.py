"""Spin-wave metric solve (sunny_geneig_launch_sigma): Sigma u = lambda S u
with Sigma = diag(I_{n/2}, -I_{n/2}) implied, S the positive-definite BdG
dynamical matrix (the call pattern of Sunny's linear spin-wave code).

Checked through the C ABI against LAPACK zhegv on the explicit pencil
(Sigma, S), with the FP64 tolerances of the other parity tests (eigenvalues
within 1e-12 ||Sigma||_2, residual <= 1e-12, ||U^H S U - I|| <= 1e-12, the
info codes identical), in every execution regime, plus the +-pairing of
the spectrum (n/2 eigenvalues of each sign) and the argument checks.
"""
import numpy as np
import pytest

from oracle import zhegv_batch
from sunny_gen_eigensolver_b200 import accuracy, generators

pytestmark = pytest.mark.gpu


def sigma_solve(S, solver=None):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    batch, n, _ = S.shape
    St = to_colmajor(torch.from_numpy(np.ascontiguousarray(S)).cuda())
    W = torch.full((batch, n), 7.0, dtype=torch.float64, device="cuda")
    U = torch.full((batch, n, n), 7.0 + 7.0j, dtype=torch.complex128, device="cuda")
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    own = solver is None
    s = Solver(n) if own else solver
    try:
        s.launch_sigma(St, W, U, info)
        torch.cuda.synchronize()
    finally:
        if own:
            s.close()
    return W.cpu().numpy(), U.transpose(-1, -2).cpu().numpy(), info.cpu().numpy()


@pytest.mark.parametrize("n", [2, 12, 54, 64, 72, 108, 162])
def test_sigma_matches_zhegv(cuda, n):
    H, S = generators.sigma_metric_problems(n, 6, seed=900 + n)
    W, U, info = sigma_solve(S)
    Wr, Ur, ir = zhegv_batch(H, S)
    assert np.array_equal(info, ir) and (ir == 0).all()
    assert accuracy.eig_err_rel(H, W, Wr).max() <= 1e-12
    assert accuracy.residual(H, S, W, U).max() <= 1e-12
    assert accuracy.s_orth(S, U).max() <= 1e-12
    assert (np.diff(W, axis=-1) >= 0).all()
    assert ((W > 0).sum(axis=1) == n // 2).all()


def test_sigma_non_pd_info_and_nan_outputs(cuda):
    n = 54
    H, S = generators.sigma_metric_problems(n, 4, seed=77)
    S[2] = np.eye(n)
    S[2, 9, 9] = -1.0                      # leading minor 10 fails: info = n + 10
    W, U, info = sigma_solve(S)
    _, _, ir = zhegv_batch(H, S)
    assert np.array_equal(info, ir) and info[2] == n + 10
    assert np.isnan(W[2]).all() and np.isnan(U[2]).all()
    ok = info == 0
    assert accuracy.residual(H[ok], S[ok], W[ok], U[ok]).max() <= 1e-12


def test_sigma_rejects_odd_n(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, _native as nat
    with Solver(9) as s:
        S = torch.zeros((1, 9, 9), dtype=torch.complex128, device="cuda")
        W = torch.zeros((1, 9), dtype=torch.float64, device="cuda")
        info = torch.zeros((1,), dtype=torch.int32, device="cuda")
        with pytest.raises(RuntimeError, match="even"):
            s.launch_sigma(S, W, S.clone(), info)
        L = nat.load()
        assert L.sunny_geneig_launch_sigma(None, 0, 0, 0, 0, 1, 0) == nat.STATUS_INVALID_ARG
