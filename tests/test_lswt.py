"""Spin-wave front end of the fused assembly (sunny_gen_eigensolver_b200.lswt)
and its oracle (oracle/fourier.py), on the CPU.

The convention of the dynamical matrix is pinned to two analytic linear
spin-wave dispersions (k = 2 pi q, q in reciprocal-lattice units):
  * Heisenberg ferromagnetic chain, coupling J < 0, field h along the
    moments: omega(k) = 2|J|S(1 - cos k) + h;
  * Heisenberg antiferromagnetic chain (two-site cell, sites at 0 and 1/2),
    J > 0, staggered field h along each moment:
    omega(k) = sqrt((2JS + h)^2 - (2JS cos(k/2))^2), twice degenerate.
"""
import ctypes

import numpy as np
import pytest

from oracle import fourier
from sunny_gen_eigensolver_b200 import lswt
from sunny_gen_eigensolver_b200 import _native as nat


def fm_chain(J=-1.0, S=1.5, h=0.3):
    return lswt.SpinModel(spins=[S], directions=[[0, 0, 1]], bonds=[(0, 0, [1, 0, 0], J * np.eye(3))],
                          fields=[[0, 0, h]])


def afm_chain(J=1.0, S=1.0, h=0.2):
    bonds = [(0, 1, [0, 0, 0], J * np.eye(3)), (1, 0, [1, 0, 0], J * np.eye(3))]
    return lswt.SpinModel(spins=[S, S], directions=[[0, 0, 1], [0, 0, -1]], bonds=bonds,
                          fields=[[0, 0, h], [0, 0, -h]])


def dyn(model, q):
    rows, cols, coef, disp = lswt.fourier_terms(model)
    return fourier.assemble(model.n, rows, cols, coef, disp, q)


def test_ferromagnetic_chain_dispersion():
    J, S, h = -1.0, 1.5, 0.3
    q = np.zeros((9, 3))
    q[:, 0] = np.linspace(0.0, 0.5, 9)
    w = fourier.magnon_energies(dyn(fm_chain(J, S, h), q))[:, 0]
    k = 2 * np.pi * q[:, 0]
    np.testing.assert_allclose(w, 2 * abs(J) * S * (1 - np.cos(k)) + h, rtol=0, atol=1e-12)


def test_antiferromagnetic_chain_dispersion():
    J, S, h = 1.0, 1.0, 0.2
    q = np.zeros((7, 3))
    q[:, 0] = np.linspace(0.0, 0.5, 7)
    w = fourier.magnon_energies(dyn(afm_chain(J, S, h), q))
    k = 2 * np.pi * q[:, 0]
    ref = np.sqrt((2 * J * S + h) ** 2 - (2 * J * S * np.cos(k / 2)) ** 2)
    np.testing.assert_allclose(w, np.stack([ref, ref], axis=1), rtol=0, atol=1e-12)


def test_dispersion_independent_of_local_frame():
    """Rotating the whole ordered state (directions, fields and exchange
    together) leaves the spectrum unchanged: the local frames are a gauge."""
    rng = np.random.default_rng(1)
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    R *= np.sign(np.linalg.det(R))
    m0 = afm_chain()
    m1 = lswt.SpinModel(spins=m0.spins, directions=[R @ np.asarray(d) for d in m0.directions],
                        bonds=[(a, b, d, R @ J @ R.T) for a, b, d, J in m0.bonds],
                        fields=[R @ np.asarray(f) for f in m0.fields])
    q = rng.uniform(-0.5, 0.5, size=(5, 3))
    np.testing.assert_allclose(fourier.magnon_energies(dyn(m0, q)), fourier.magnon_energies(dyn(m1, q)),
                               rtol=0, atol=1e-12)


def test_random_model_hermitian_positive_definite():
    model = lswt.random_model(27, 120, seed=5)
    q = np.random.default_rng(2).uniform(-0.5, 0.5, size=(16, 3))
    S = dyn(model, q)
    assert S.shape == (16, 54, 54)
    np.testing.assert_allclose(S, np.conj(np.swapaxes(S, -1, -2)), rtol=0, atol=1e-13)
    assert np.linalg.eigvalsh(S).min() > 0.1


def test_pack_terms_lower_triangle_round_trip():
    model = lswt.random_model(6, 20, seed=3)
    rows, cols, coef, disp = lswt.fourier_terms(model)
    n = model.n
    start, c, d = lswt.pack_terms(n, rows, cols, coef, disp)
    assert start.dtype == np.int32 and start.shape == (n * n + 1,) and start[0] == 0
    assert (np.diff(start) >= 0).all() and start[-1] == c.shape[0] == d.shape[0]
    q = np.random.default_rng(4).uniform(-0.5, 0.5, size=(3, 3))
    full = fourier.assemble(n, rows, cols, coef, disp, q)
    # rebuild the lower triangle from the packed table, entry by entry
    e = np.repeat(np.arange(n * n), np.diff(start))
    r, cc = e % n, e // n
    assert (r >= cc).all()
    low = fourier.assemble(n, r, cc, c, d, q)
    il = np.tril_indices(n)
    np.testing.assert_allclose(low[:, il[0], il[1]], full[:, il[0], il[1]], rtol=0, atol=1e-13)
    with pytest.raises(ValueError):
        lswt.pack_terms(n, rows + n, cols, coef, disp)


def test_fourier_entry_points_reject_null_handle():
    L = nat.load()
    st = L.sunny_geneig_launch_fourier_sigma(None, 0, 0, 0, 0, 0, 0, 0, 0, 4, 0)
    assert st == nat.STATUS_INVALID_ARG and "NULL" in nat.last_error()
    st = L.sunny_geneig_launch_fourier_sigma_intensity(None, 0, 0, 0, 0, 0, 0, 0, 0, 8, ctypes.c_double(0.1),
                                                      0, 0, 0, 4, 0)
    assert st == nat.STATUS_INVALID_ARG and "NULL" in nat.last_error()


def test_random_model_is_seeded_and_packs_empty_tables():
    a = lswt.fourier_terms(lswt.random_model(5, 12, seed=7))
    b = lswt.fourier_terms(lswt.random_model(5, 12, seed=7))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    start, c, d = lswt.pack_terms(6, np.zeros(0, int), np.zeros(0, int), np.zeros(0, complex), np.zeros((0, 3)))
    assert start.shape == (37,) and (start == 0).all() and c.shape == (0,) and d.shape == (0, 3)
