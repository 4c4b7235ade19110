"""The oracle, pinned against the reference's golden fixtures (CPU only)."""
import hashlib

import numpy as np
import pytest

from oracle import chain_batch, fixtures, reduce_batch, zhegv_batch, zheev_batch, zpotrf_batch
from sunny_gen_eigensolver_b200 import accuracy


def _colmajor_bytes(M):
    return np.ascontiguousarray(M.transpose(0, 2, 1)).tobytes()


def test_generator_reproduces_every_fixture(golden):
    assert len(golden) == 15
    for name, rec in golden.items():
        H, S = fixtures.generate(rec["n"], rec["batch"], rec["seed"], rec["mode"])
        assert hashlib.sha256(_colmajor_bytes(H)).digest() == rec["sha_H"], name
        assert hashlib.sha256(_colmajor_bytes(S)).digest() == rec["sha_S"], name


@pytest.mark.parametrize("name", ["n16_b8_s42_random", "n32_b8_s42_nearid", "n54_b8_s42_random",
                                  "n54_b8_s42_nearid", "n54_b32_s123_random", "n64_b8_s42_random",
                                  "n96_b8_s42_nearid", "n128_b8_s42_random"])
def test_zhegv_matches_fixture_eigenvalues(golden, name):
    rec = golden[name]
    H, S = fixtures.generate(rec["n"], rec["batch"], rec["seed"], rec["mode"])
    W, U, info = zhegv_batch(H, S)
    assert (info == 0).all()
    # the reference's own acceptance metric and tolerance (tests/unified/test_n54.cpp:33-35)
    assert accuracy.eig_rel_ref(W, rec["W"]).max() < 1e-12
    assert accuracy.eig_err_rel(H, W, rec["W"]).max() < 1e-13
    assert accuracy.residual(H, S, W, U).max() < 1e-13
    assert accuracy.s_orth(S, U).max() < 1e-12
    if "U2" in rec:
        ph = accuracy.phase_err(S[:2], U[:2], rec["U2"], rec["W"][:2])
        assert ph.max() < 1e-10


def test_chain_restatement_matches_zhegv(golden):
    rec = golden["n54_b8_s42_random"]
    H, S = fixtures.generate(rec["n"], rec["batch"], rec["seed"], rec["mode"])
    W, U, info = chain_batch(H, S)
    Wr, Ur, _ = zhegv_batch(H, S)
    assert (info == 0).all()
    assert accuracy.eig_err_rel(H, W, Wr).max() < 1e-13
    assert accuracy.residual(H, S, W, U).max() < 1e-13
    assert accuracy.s_orth(S, U).max() < 1e-12


def test_stage_oracles_consistent(golden):
    rec = golden["n32_b8_s42_random"]
    H, S = fixtures.generate(rec["n"], rec["batch"], rec["seed"], rec["mode"])
    L, info = zpotrf_batch(S)
    assert (info == 0).all()
    assert np.abs(L @ np.conj(np.swapaxes(L, -1, -2)) - S).max() < 1e-12 * np.abs(S).max()
    C, _, _ = reduce_batch(H, S)
    assert np.abs(C - np.conj(np.swapaxes(C, -1, -2))).max() < 1e-12 * np.abs(C).max()
    Wc, V = zheev_batch(C)
    assert np.abs(Wc - rec["W"]).max() < 1e-12 * np.abs(rec["W"]).max()


def test_zhegv_info_for_non_pd_S():
    rng = np.random.default_rng(7)
    n = 6
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    H = (A + A.conj().T)[None]
    S = np.eye(n, dtype=np.complex128)[None].copy()
    S[0, 3, 3] = -1.0          # leading minor of order 4 is not PD
    _, _, info = zhegv_batch(H, S)
    assert info[0] == n + 4


def test_geig_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    H = rng.standard_normal((2, 3, 3)) + 1j * rng.standard_normal((2, 3, 3))
    S = rng.standard_normal((2, 3, 3)) + 1j * rng.standard_normal((2, 3, 3))
    W = rng.standard_normal((2, 3))
    U = rng.standard_normal((2, 3, 3)) + 1j * rng.standard_normal((2, 3, 3))
    p = tmp_path / "x.bin"
    fixtures.write_geig(p, H, S, W, U, seed=5)
    r = fixtures.read_geig(p)
    assert r["seed"] == 5 and np.array_equal(r["H"], H) and np.array_equal(r["U"], U) and np.array_equal(r["W"], W)
