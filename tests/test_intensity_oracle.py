"""The intensity restatement (oracle/intensity.py) on the CPU: the
Bogoliubov vectors it forms are para-unitary and diagonalise the dynamical
matrix, and the broadened spectrum integrates to the summed intensities."""
import numpy as np
from scipy.linalg import lapack

from oracle.intensity import sigma_intensities, sigma_matrix
from sunny_gen_eigensolver_b200 import generators


def test_bogoliubov_normalisation_and_sum_rule():
    n, batch = 12, 3
    _, D = generators.sigma_metric_problems(n, batch, seed=4)
    rng = np.random.default_rng(4)
    O = rng.standard_normal((batch, 3, n)) + 1j * rng.standard_normal((batch, 3, n))
    q = np.tile(np.array([0.0, 0.0, 1.0]), (batch, 1))
    E = np.linspace(-5.0, 40.0, 20001)
    W, om, I, spec, info = sigma_intensities(D, O, q, E, 0.05)
    assert (info == 0).all() and (om > 0).all() and (I >= -1e-12).all()
    # para-unitarity of the positive modes: t^H Sigma t = 1, t^H D t = omega
    w, U, _ = lapack.zhegv(sigma_matrix(n), D[0], itype=1, jobz="V", uplo="L")
    pos = w > 0
    T = U[:, pos] / np.sqrt(w[pos])
    assert np.allclose(np.conj(T.T) @ sigma_matrix(n) @ T, np.eye(pos.sum()), atol=1e-10)
    assert np.allclose(np.diag(np.conj(T.T) @ D[0] @ T).real, 1.0 / w[pos], rtol=1e-10)
    # the Gaussian is normalised: the spectrum integrates to sum_k I_k
    integral = np.trapezoid(spec, E, axis=1)
    assert np.allclose(integral, I.sum(axis=1), rtol=1e-6)
