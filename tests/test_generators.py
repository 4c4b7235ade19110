"""Workload generators and accuracy measures (CPU only)."""
import numpy as np
import pytest

from sunny_gen_eigensolver_b200 import accuracy, generators


@pytest.mark.parametrize("kappa", [1e1, 1e2, 1e5])
def test_baseline_distribution(kappa):
    H, S = generators.baseline_problems(54, 16, seed=20261204, kappa=kappa)
    assert H.shape == (16, 54, 54) and S.shape == (16, 54, 54)
    assert np.array_equal(H, np.conj(np.swapaxes(H, -1, -2)))
    assert np.array_equal(S, np.conj(np.swapaxes(S, -1, -2)))
    ev = np.linalg.eigvalsh(H)
    assert np.allclose(ev[:, 0] / ev[:, -1], 0.1, rtol=1e-9)
    es = np.linalg.eigvalsh(S)
    assert es.min() > 1.0 - 1e-9 and es.max() < kappa * (1 + 1e-9)
    H2, S2 = generators.baseline_problems(54, 16, seed=20261204, kappa=kappa)
    assert np.array_equal(H, H2) and np.array_equal(S, S2)


def test_bdg_block_structure():
    H, _ = generators.baseline_problems(12, 4, seed=3)
    m = 6
    A, B = H[:, :m, :m], H[:, :m, m:]
    assert np.allclose(H[:, m:, m:], np.conj(A)) and np.allclose(H[:, m:, :m], np.conj(B))
    assert np.allclose(B, np.swapaxes(B, -1, -2))


def test_sigma_metric_pattern():
    H, S = generators.sigma_metric_problems(8, 3, seed=1)
    assert np.array_equal(H[0], np.diag([1, 1, 1, 1, -1, -1, -1, -1]).astype(complex))
    assert np.linalg.eigvalsh(S).min() > 0


def test_accuracy_measures_on_exact_solution():
    from oracle import zhegv_batch
    H, S = generators.baseline_problems(16, 4, seed=9)
    W, U, _ = zhegv_batch(H, S)
    assert accuracy.residual(H, S, W, U).max() < 1e-13
    assert accuracy.s_orth(S, U).max() < 1e-12
    assert accuracy.eig_err_rel(H, W, W).max() == 0.0
    assert accuracy.phase_err(S, U, U * np.exp(1j * 0.3), W).max() < 1e-12
    assert accuracy.subspace_err(S, U, U, W, 1e-6).max() < 1e-12
    assert accuracy.clusters(np.array([0.0, 1e-9, 1.0, 2.0, 2.0]), 1e-6) == [(0, 2), (2, 3), (3, 5)]
