"""Fused dynamical-matrix assembly on the device
(sunny_geneig_launch_fourier_sigma[_intensity]) against its CPU oracle:
oracle/fourier.py assembles S(q) from the same terms, LAPACK zhegv solves
the metric pencil H = diag(I, -I), and oracle/intensity.py reduces it to
spectra. Tolerances: eigenvalues within 1e-12 ||Sigma||_2 = 1e-12 (the
assembly adds O(1e-16) relative rounding per term), residual and
S-orthonormality 1e-12 against the oracle-assembled S, spectra within 1e-9
of their largest value, magnon energies of the analytic chains within
1e-12 relative."""
import numpy as np
import pytest

from oracle import fourier, zhegv_batch
from oracle.intensity import sigma_intensities
from sunny_gen_eigensolver_b200 import accuracy, lswt

pytestmark = pytest.mark.gpu


def _device_case(model, q):
    import torch
    rows, cols, coef, disp = lswt.fourier_terms(model)
    n = model.n
    start, c, d = lswt.pack_terms(n, rows, cols, coef, disp)
    S = fourier.assemble(n, rows, cols, coef, disp, q)
    dev = torch.device("cuda")
    terms = (torch.from_numpy(start).to(dev), torch.from_numpy(c).to(dev), torch.from_numpy(d).to(dev))
    return S, terms, torch.from_numpy(np.ascontiguousarray(q, dtype=np.float64)).to(dev)


def _solve(n, terms, qd):
    import torch
    from sunny_gen_eigensolver_b200 import Solver
    batch = qd.shape[0]
    W = torch.empty((batch, n), dtype=torch.float64, device=qd.device)
    U = torch.empty((batch, n, n), dtype=torch.complex128, device=qd.device)
    info = torch.empty((batch,), dtype=torch.int32, device=qd.device)
    with Solver(n) as s:
        s.launch_fourier_sigma(terms, qd, W, U, info)
        torch.cuda.synchronize()
    return W.cpu().numpy(), U.transpose(-1, -2).cpu().numpy(), info.cpu().numpy()


@pytest.mark.parametrize("m,bonds", [(8, 30), (12, 40), (27, 120), (30, 140)])
def test_fourier_sigma_matches_oracle(cuda, m, bonds):
    model = lswt.random_model(m, bonds, seed=40 + m)
    q = np.random.default_rng(m).uniform(-0.5, 0.5, size=(96, 3))
    S, terms, qd = _device_case(model, q)
    n = model.n
    H = np.broadcast_to(np.diag(np.r_[np.ones(m), -np.ones(m)]).astype(np.complex128), S.shape).copy()
    W, U, info = _solve(n, terms, qd)
    Wr, _, ir = zhegv_batch(H, S)
    assert (info == 0).all() and (ir == 0).all()
    assert np.abs(W - Wr).max() <= 1e-12
    assert accuracy.residual(H, S, W, U).max() <= 1e-12
    assert accuracy.s_orth(S, U).max() <= 1e-12
    assert (np.diff(W, axis=-1) >= 0).all()


def test_fourier_sigma_analytic_chains(cuda):
    for model, ref in (
        (lswt.SpinModel(spins=[1.5], directions=[[0, 0, 1]], bonds=[(0, 0, [1, 0, 0], -1.0 * np.eye(3))],
                        fields=[[0, 0, 0.3]]),
         lambda k: np.stack([2 * 1.5 * (1 - np.cos(k)) + 0.3], axis=1)),
        (lswt.SpinModel(spins=[1.0, 1.0], directions=[[0, 0, 1], [0, 0, -1]],
                        bonds=[(0, 1, [0, 0, 0], np.eye(3)), (1, 0, [1, 0, 0], np.eye(3))],
                        fields=[[0, 0, 0.2], [0, 0, -0.2]]),
         lambda k: np.repeat(np.sqrt(2.2 ** 2 - (2 * np.cos(k / 2)) ** 2)[:, None], 2, axis=1)),
    ):
        q = np.zeros((33, 3))
        q[:, 0] = np.linspace(-0.5, 0.5, 33)
        _, terms, qd = _device_case(model, q)
        W, _, info = _solve(model.n, terms, qd)
        assert (info == 0).all()
        omega = np.sort(1.0 / W[:, W.shape[1] // 2:], axis=1)    # positive eigenvalues -> energies
        want = ref(2 * np.pi * q[:, 0])
        np.testing.assert_allclose(omega, want, rtol=1e-12, atol=0)


def test_fourier_intensity_matches_oracle(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver
    m = 27
    model = lswt.random_model(m, 120, seed=9)
    n, batch = model.n, 40
    rng = np.random.default_rng(10)
    q = rng.uniform(-0.5, 0.5, size=(batch, 3))
    S, terms, qd = _device_case(model, q)
    O = rng.standard_normal((batch, 3, n)) + 1j * rng.standard_normal((batch, 3, n))
    qh = rng.standard_normal((batch, 3))
    qh /= np.linalg.norm(qh, axis=1, keepdims=True)
    _, om, _, _, _ = sigma_intensities(S, O, qh, np.linspace(0.0, 1.0, 4), 0.1)
    emax = np.nanmax(om) * 1.2
    E = np.linspace(0.0, emax, 160)
    fwhm = emax / 40
    Wr, _, _, spec_r, ir = sigma_intensities(S, O, qh, E, fwhm)
    dev = qd.device
    Oc = torch.from_numpy(np.ascontiguousarray(np.swapaxes(O, 1, 2))).to(dev)
    W = torch.empty((batch, n), dtype=torch.float64, device=dev)
    spec = torch.empty((batch, len(E)), dtype=torch.float64, device=dev)
    info = torch.empty((batch,), dtype=torch.int32, device=dev)
    with Solver(n) as s:
        s.launch_fourier_sigma_intensity(terms, qd, Oc, torch.from_numpy(qh).to(dev), torch.from_numpy(E).to(dev),
                                         fwhm, W, spec, info)
        torch.cuda.synchronize()
    W, spec, info = W.cpu().numpy(), spec.cpu().numpy(), info.cpu().numpy()
    assert (info == 0).all() and (ir == 0).all()
    assert np.abs(W - Wr).max() <= 1e-12
    scale = np.abs(spec_r).max(axis=1, keepdims=True)
    assert (np.abs(spec - spec_r) / scale).max() <= 1e-9


def test_fourier_rejects_unsupported(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver
    dev = torch.device("cuda")
    start = torch.zeros((72 * 72 + 1,), dtype=torch.int32, device=dev)
    coef = torch.zeros((0,), dtype=torch.complex128, device=dev)
    disp = torch.zeros((0, 3), dtype=torch.float64, device=dev)
    q = torch.zeros((1, 3), dtype=torch.float64, device=dev)
    with Solver(72) as s:                               # l2-slot regime: not supported
        W = torch.zeros((1, 72), dtype=torch.float64, device=dev)
        U = torch.zeros((1, 72, 72), dtype=torch.complex128, device=dev)
        info = torch.zeros((1,), dtype=torch.int32, device=dev)
        with pytest.raises(RuntimeError, match="smem-cta"):
            s.launch_fourier_sigma((start, coef, disp), q, W, U, info)


def test_fourier_empty_terms_give_non_pd_info(cuda):
    """No terms: S(q) = 0, whose first leading minor is not positive
    definite: info = n + 1 and NaN outputs, as zhegv reports."""
    import torch
    n = 8
    dev = torch.device("cuda")
    start = torch.zeros((n * n + 1,), dtype=torch.int32, device=dev)
    coef = torch.zeros((0,), dtype=torch.complex128, device=dev)
    disp = torch.zeros((0, 3), dtype=torch.float64, device=dev)
    q = torch.zeros((3, 3), dtype=torch.float64, device=dev)
    W, U, info = _solve(n, (start, coef, disp), q)
    assert (info == n + 1).all() and np.isnan(W).all() and np.isnan(U).all()
