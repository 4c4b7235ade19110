"""Spin-wave intensities on the device (sunny_geneig_launch_sigma_intensity)
against the CPU restatement oracle/intensity.py (LAPACK zhegv on the metric
pencil, Bogoliubov normalisation, perpendicular projection, Gaussian
broadening). Tolerances: eigenvalues within 1e-12 ||Sigma||_2 = 1e-12; the
spectrum within 1e-9 of its largest value (the intensities are quadratic in
the eigenvectors, whose rounding errors are ~1e-14 relative; degenerate
modes enter only through their sum, which is invariant)."""
import numpy as np
import pytest

from oracle.intensity import sigma_intensities
from sunny_gen_eigensolver_b200 import generators

pytestmark = pytest.mark.gpu


def _case(n, batch, seed):
    _, D = generators.sigma_metric_problems(n, batch, seed=seed)
    rng = np.random.default_rng(seed)
    O = rng.standard_normal((batch, 3, n)) + 1j * rng.standard_normal((batch, 3, n))
    q = rng.standard_normal((batch, 3))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return D, O, q


@pytest.mark.parametrize("n", [8, 18, 54])
def test_intensity_matches_oracle(cuda, n):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    batch = 12
    D, O, q = _case(n, batch, seed=300 + n)
    D[5] = np.eye(n)
    D[5, 3, 3] = -1.0                                   # non-PD: info = n + 4, NaN outputs
    _, om, _, _, _ = sigma_intensities(D, O, q, np.linspace(0.0, 1.0, 4), 0.1)
    emax = np.nanmax(om) * 1.2
    E = np.linspace(0.0, emax, 200)
    fwhm = emax / 40
    Wr, om, I, spec_r, ir = sigma_intensities(D, O, q, E, fwhm)
    dev = torch.device("cuda")
    Dc = to_colmajor(torch.from_numpy(D).to(dev))
    Oc = torch.from_numpy(np.ascontiguousarray(np.swapaxes(O, 1, 2))).to(dev)   # (batch, n, 3): column-major 3 x n
    qd = torch.from_numpy(q).to(dev)
    Ed = torch.from_numpy(E).to(dev)
    W = torch.empty((batch, n), dtype=torch.float64, device=dev)
    spec = torch.empty((batch, len(E)), dtype=torch.float64, device=dev)
    info = torch.empty((batch,), dtype=torch.int32, device=dev)
    with Solver(n) as s:
        s.launch_sigma_intensity(Dc, Oc, qd, Ed, fwhm, W, spec, info)
        torch.cuda.synchronize()
    W, spec, info = W.cpu().numpy(), spec.cpu().numpy(), info.cpu().numpy()
    assert np.array_equal(info, ir) and ir[5] == n + 4
    assert np.isnan(W[5]).all() and np.isnan(spec[5]).all()
    ok = ir == 0
    assert np.abs(W[ok] - Wr[ok]).max() <= 1e-12
    scale = np.abs(spec_r[ok]).max(axis=1, keepdims=True)
    assert (np.abs(spec[ok] - spec_r[ok]) / scale).max() <= 1e-9
    assert (spec[ok] >= -1e-12 * scale).all()


def test_intensity_rejects_unsupported(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver
    dev = torch.device("cuda")
    n = 72
    with Solver(n) as s:                                # l2-slot regime: not supported
        S = torch.zeros((1, n, n), dtype=torch.complex128, device=dev)
        O = torch.zeros((1, n, 3), dtype=torch.complex128, device=dev)
        q = torch.zeros((1, 3), dtype=torch.float64, device=dev)
        E = torch.zeros((4,), dtype=torch.float64, device=dev)
        W = torch.zeros((1, n), dtype=torch.float64, device=dev)
        sp = torch.zeros((1, 4), dtype=torch.float64, device=dev)
        info = torch.zeros((1,), dtype=torch.int32, device=dev)
        with pytest.raises(RuntimeError, match="smem-cta"):
            s.launch_sigma_intensity(S, O, q, E, 0.1, W, sp, info)
