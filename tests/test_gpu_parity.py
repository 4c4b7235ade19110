"""GPU parity: libsunny_geneig.so (through its C ABI) against the oracle.

Tolerances (FP64 throughout):
  * eigenvalues: |W - W_zhegv| <= 1e-12 * ||H||_2, and the reference's own
    acceptance metric eig_rel < 1e-10 (tests/unified/test_n54.cpp:33-35)
  * residual ||H U - S U diag(W)||_F / (||H||_2 ||U||_2) <= 1e-12
  * S-orthonormality max |U^H S U - I| <= 1e-12
  * eigenvector phase vs the fixture's zhegvd vectors 1 - |u^H S u_ref| < 1e-10
    for eigenvalues with gap >= 1e-6 (test_n54.cpp:148-162)
  * info codes identical to LAPACK zhegv's, bit for bit.
Eigenvectors are compared by residual and subspace, never by element.
"""
import numpy as np
import pytest

from oracle import fixtures, reduce_batch, zhegv_batch, zpotrf_batch, zheev_batch
from sunny_gen_eigensolver_b200 import accuracy, generators

pytestmark = pytest.mark.gpu

EIG_TOL = 1e-12
RES_TOL = 1e-12
ORTH_TOL = 1e-12


def gpu_solve(H, S, stage=4, solver=None):
    import torch
    from sunny_gen_eigensolver_b200 import solve
    Ht = torch.from_numpy(np.ascontiguousarray(H)).cuda()
    St = torch.from_numpy(np.ascontiguousarray(S)).cuda()
    W, U, info = solve(Ht, St, solver=solver, stage=stage)
    return W.cpu().numpy(), U.cpu().numpy(), info.cpu().numpy()


def check_against_zhegv(H, S, W, U, info, eig_tol=EIG_TOL, res_tol=RES_TOL, orth_tol=ORTH_TOL):
    Wr, Ur, ir = zhegv_batch(H, S)
    assert np.array_equal(info, ir)
    ok = ir == 0
    if not ok.any():
        return
    e = accuracy.eig_err_rel(H[ok], W[ok], Wr[ok])
    r = accuracy.residual(H[ok], S[ok], W[ok], U[ok])
    o = accuracy.s_orth(S[ok], U[ok])
    assert e.max() <= eig_tol, e.max()
    assert r.max() <= res_tol, r.max()
    assert o.max() <= orth_tol, o.max()
    assert (np.diff(W[ok], axis=-1) >= 0).all()
    return e, r, o


@pytest.mark.parametrize("name", ["n16_b8_s42_random", "n16_b8_s42_nearid", "n32_b8_s42_random",
                                  "n32_b8_s42_nearid", "n48_b8_s42_random", "n48_b8_s42_nearid",
                                  "n54_b8_s42_random", "n54_b8_s42_nearid", "n54_b32_s123_random",
                                  "n64_b8_s42_random", "n64_b8_s42_nearid", "n96_b8_s42_random",
                                  "n96_b8_s42_nearid", "n128_b8_s42_random", "n128_b8_s42_nearid"])
def test_reference_fixtures(cuda, golden, name):
    rec = golden[name]
    H, S = fixtures.generate(rec["n"], rec["batch"], rec["seed"], rec["mode"])
    W, U, info = gpu_solve(H, S)
    assert (info == 0).all()
    assert accuracy.eig_rel_ref(W, rec["W"]).max() < 1e-10
    check_against_zhegv(H, S, W, U, info)
    if "U2" in rec:
        assert accuracy.phase_err(S[:2], U[:2], rec["U2"], rec["W"][:2]).max() < 1e-10


@pytest.mark.parametrize("n", [2, 4, 12, 18, 24, 50, 54, 56, 72, 80, 108, 128])
def test_baseline_generator_sizes(cuda, n):
    H, S = generators.baseline_problems(n, 16, seed=20261203 + n)
    W, U, info = gpu_solve(H, S)
    check_against_zhegv(H, S, W, U, info)


@pytest.mark.parametrize("n", [162, 216, 384])
def test_large_sizes_l2_slot(cuda, n):
    H, S = generators.baseline_problems(n, 2, seed=97 + n)
    W, U, info = gpu_solve(H, S)
    check_against_zhegv(H, S, W, U, info)


@pytest.mark.parametrize("n", [1, 3, 5, 7, 33, 55, 61, 97, 129])
def test_odd_sizes(cuda, n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((5, n, n)) + 1j * rng.standard_normal((5, n, n))
    H = A + np.conj(np.swapaxes(A, -1, -2))
    B = rng.standard_normal((5, n, n)) + 1j * rng.standard_normal((5, n, n))
    S = B @ np.conj(np.swapaxes(B, -1, -2)) + n * np.eye(n)
    W, U, info = gpu_solve(H, S)
    check_against_zhegv(H, S, W, U, info)


def test_sigma_metric_indefinite_H(cuda):
    H, S = generators.sigma_metric_problems(54, 8, seed=11)
    W, U, info = gpu_solve(H, S)
    check_against_zhegv(H, S, W, U, info)
    # eigenvalues come in +-1/omega pairs with n/2 of each sign
    assert ((W > 0).sum(axis=1) == 27).all()


def test_degenerate_clusters(cuda):
    n = 24
    rng = np.random.default_rng(5)
    # S = I, H with 3-fold repeated eigenvalues in a random unitary basis
    X = rng.standard_normal((4, n, n)) + 1j * rng.standard_normal((4, n, n))
    Q, _ = np.linalg.qr(X)
    lam = np.repeat(np.arange(n // 3, dtype=float), 3)
    H = (Q * lam[None, None, :]) @ np.conj(np.swapaxes(Q, -1, -2))
    H = 0.5 * (H + np.conj(np.swapaxes(H, -1, -2)))
    S = np.broadcast_to(np.eye(n, dtype=np.complex128), H.shape).copy()
    W, U, info = gpu_solve(H, S)
    check_against_zhegv(H, S, W, U, info)
    Wr, Ur, _ = zhegv_batch(H, S)
    assert accuracy.subspace_err(S, U, Ur, Wr, 1e-6).max() < 1e-10
    # all-equal eigenvalues: H = 2 I
    H2 = 2.0 * S
    W2, U2, info2 = gpu_solve(H2, S)
    assert (info2 == 0).all() and np.allclose(W2, 2.0, atol=1e-14)
    assert accuracy.s_orth(S, U2).max() < 1e-13


def test_non_positive_definite_S_info_codes(cuda):
    n = 12
    rng = np.random.default_rng(2)
    A = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    H = A + np.conj(np.swapaxes(A, -1, -2))
    S = np.broadcast_to(np.eye(n, dtype=np.complex128), (n, n, n)).copy()
    for b in range(n):
        S[b, b, b] = -1.0 if b % 2 else 0.0   # leading minor b+1 not PD
    S[3] = np.eye(n)                           # this one is fine
    W, U, info = gpu_solve(H, S)
    _, _, ir = zhegv_batch(H, S)
    assert np.array_equal(info, ir)
    bad = info != 0
    assert np.isnan(W[bad]).all() and np.isnan(U[bad]).all()
    assert info[3] == 0 and not np.isnan(W[3]).any()


@pytest.mark.parametrize("n", [2, 16, 54, 72, 108])
def test_nan_input_info_matches_zhegv(cuda, n):
    """NaN in H: the info code is zhegv's (n - 1 for n >= 3, 0 for n <= 2:
    its tridiagonal QR counts every off-diagonal as unconverged) and W and U
    are NaN; the other problems of the batch are unaffected."""
    H, S = generators.baseline_problems(n, 3, seed=1)
    H[1, 0, 1] = np.nan
    H[1, 1, 0] = np.nan
    W, U, info = gpu_solve(H, S)
    _, _, ir = zhegv_batch(H, S)
    assert np.array_equal(info, ir), (info, ir)
    assert info[1] == (n - 1 if n >= 3 else 0)
    assert np.isnan(W[1]).all() and np.isnan(U[1]).all()
    check_against_zhegv(H[[0, 2]], S[[0, 2]], W[[0, 2]], U[[0, 2]], info[[0, 2]])


@pytest.mark.parametrize("n", [54, 108])
def test_stage_cholesky(cuda, n):
    H, S = generators.baseline_problems(n, 6, seed=3)
    _, U, info = gpu_solve(H, S, stage=1)
    L, ir = zpotrf_batch(S)
    assert (info == 0).all() and (ir == 0).all()
    assert np.abs(U - L).max() <= 1e-12 * np.abs(L).max()


@pytest.mark.parametrize("n", [54, 108])
def test_stage_reduce(cuda, n):
    H, S = generators.baseline_problems(n, 6, seed=4)
    _, C, info = gpu_solve(H, S, stage=2)
    Cr, _, _ = reduce_batch(H, S)
    assert (info == 0).all()
    assert np.abs(C - Cr).max() <= 1e-11 * np.abs(Cr).max()
    assert np.array_equal(C, np.conj(np.swapaxes(C, -1, -2)))


@pytest.mark.parametrize("n", [54, 108])
def test_stage_reduce_eig(cuda, n):
    H, S = generators.baseline_problems(n, 6, seed=5)
    W, V, info = gpu_solve(H, S, stage=3)
    Cr, _, _ = reduce_batch(H, S)
    Wr, _ = zheev_batch(Cr)
    assert (info == 0).all()
    assert accuracy.eig_err_rel(Cr, W, Wr).max() < 1e-12
    I = np.broadcast_to(np.eye(n), Cr.shape)
    assert accuracy.residual(Cr, I, W, V).max() < 1e-12
    assert accuracy.s_orth(I, V).max() < 1e-12


def test_batch_edges_and_determinism(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    n = 54
    H, S = generators.baseline_problems(n, 37, seed=8)
    with Solver(n) as s:
        assert s.regime == "smem-cta" and s.block_dim_x > 0 and s.shared_mem_bytes > 0
        Ht = to_colmajor(torch.from_numpy(H).cuda())
        St = to_colmajor(torch.from_numpy(S).cuda())
        W1, U1, i1 = s.run_kernel(Ht, St)
        W2, U2, i2 = s.run_kernel(Ht, St)
        torch.cuda.synchronize()
        assert torch.equal(W1, W2) and torch.equal(U1, U2) and torch.equal(i1, i2)
        # chunked multi-stream launch gives bit-identical results (test_streams_n54.cpp)
        W3 = torch.zeros_like(W1); U3 = torch.zeros_like(U1); i3 = torch.full_like(i1, -7)
        s.run_kernel_chunked(Ht, St, W3, U3, i3, num_streams=3, chunk_size=5)
        assert torch.equal(W1, W3) and torch.equal(U1, U3) and torch.equal(i1, i3)
        # batch 0 is a no-op
        W0 = torch.full((0, n), 7.0, dtype=torch.float64, device="cuda")
        s.launch(Ht[:0], St[:0], W0, U1[:0], i1[:0])
        # single matrix equals its slot in the batch
        Wx, Ux, ix = s.run_kernel(Ht[5:6].contiguous(), St[5:6].contiguous())
        torch.cuda.synchronize()
        assert torch.equal(Wx[0], W1[5]) and torch.equal(Ux[0], U1[5])


@pytest.mark.parametrize("n,request_,expect", [(12, 4, 4), (16, 2, 2), (16, 8, 4), (24, 2, 2), (32, 4, 2),
                                                (40, 2, 1), (54, 4, 1), (72, 4, 1)])
def test_batches_per_block(cuda, n, request_, expect):
    """batches_per_block_request > 1: several pencils per CTA (teams with their
    own barriers) where the smem-cta kernel has that form; results, info
    codes and the ragged last CTA equal the one-pencil-per-CTA launch bit for
    bit (reference: src/unified/unified_solver.cpp:1021-1042 picks BPB)."""
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    H, S = generators.baseline_problems(n, 37, seed=11)
    S[5] = np.eye(n)
    S[5, 2, 2] = -1.0                                   # info = n + 3
    Ht = to_colmajor(torch.from_numpy(H).cuda())
    St = to_colmajor(torch.from_numpy(S).cuda())
    with Solver(n, bpb_request=1) as s1, Solver(n, bpb_request=request_) as s2:
        assert s1.batches_per_block == 1
        assert s2.batches_per_block == expect
        assert s2.block_dim_x == expect * s1.block_dim_x
        W1, U1, i1 = s1.run_kernel(Ht, St)
        W2, U2, i2 = s2.run_kernel(Ht, St)
        torch.cuda.synchronize()
    assert torch.equal(i1, i2) and int(i2[5]) == n + 3
    assert torch.equal(W1.nan_to_num(7.0), W2.nan_to_num(7.0))
    assert torch.equal(U1.nan_to_num(7.0), U2.nan_to_num(7.0))
    ok = i2.cpu().numpy() == 0
    W = W2.cpu().numpy()
    U = U2.transpose(-1, -2).cpu().numpy()
    check_against_zhegv(H[ok], S[ok], W[ok], U[ok], i2.cpu().numpy()[ok])


def test_abi_errors_on_gpu(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, _native as nat
    with Solver(16) as s:
        L = nat.load()
        buf = torch.zeros(4 * 16 * 16 * 2 + 8, dtype=torch.float64, device="cuda")
        p = buf.data_ptr()
        st = L.sunny_geneig_launch(s.handle, p + 8, p, p, p, p, 1, 0)
        assert st == nat.STATUS_INVALID_ARG and "misaligned" in nat.last_error()
        st = L.sunny_geneig_launch(s.handle, 0, p, p, p, p, 1, 0)
        assert st == nat.STATUS_INVALID_ARG and "NULL" in nat.last_error()
        st = L.sunny_geneig_launch(s.handle, p, p, p, p, p, -1, 0)
        assert st == nat.STATUS_INVALID_ARG
        assert L.sunny_geneig_launch(s.handle, p, p, p, p, p, 0, 0) == nat.STATUS_OK
        assert s.path_name == "unified" and s.kernel_mode == "unified"
    with Solver(16, kernel="hybrid") as s:
        assert s.path_name == "hybrid"


def test_one_l2_slot_handle_on_two_streams(cuda):
    """A handle whose solver keeps scratch slots, launched from two streams
    back to back: the second launch must not overlap the first on the slots."""
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    n = 108
    H, S = generators.baseline_problems(n, 24, seed=5150)
    Ht, St = to_colmajor(torch.from_numpy(H).cuda()), to_colmajor(torch.from_numpy(S).cuda())
    with Solver(n) as s:
        assert s.regime == "l2-slot"
        Wr, Ur, ir = s.run_kernel(Ht, St)
        torch.cuda.synchronize()
        s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
        outs = []
        for rep in range(3):
            for st, sl in ((s1, slice(0, 12)), (s2, slice(12, 24))):
                W = torch.empty((12, n), dtype=torch.float64, device="cuda")
                U = torch.empty((12, n, n), dtype=torch.complex128, device="cuda")
                info = torch.empty((12,), dtype=torch.int32, device="cuda")
                with torch.cuda.stream(st):
                    s.launch(Ht[sl], St[sl], W, U, info, st)
                outs.append((sl, W, U, info))
        torch.cuda.synchronize()
        for sl, W, U, info in outs:
            assert torch.equal(W, Wr[sl]) and torch.equal(U, Ur[sl]) and torch.equal(info, ir[sl])


@pytest.mark.parametrize("big,small", [(64, 50), (384, 108), (80, 66)])
def test_smaller_handle_created_later_keeps_larger_working(cuda, big, small):
    """Handles for a large and then a smaller N of the same kernel are both
    usable afterwards (creating the second must not lower a launch limit the
    first one relies on)."""
    from sunny_gen_eigensolver_b200 import Solver
    s_big = Solver(big)
    s_small = Solver(small)
    try:
        for n, s in ((big, s_big), (small, s_small)):
            H, S = generators.baseline_problems(n, 2, seed=n)
            W, U, info = gpu_solve(H, S, solver=s)
            check_against_zhegv(H, S, W, U, info)
    finally:
        s_small.close()
        s_big.close()


@pytest.mark.parametrize("n,regime", [(72, "smem-wide"), (80, "smem-wide"), (64, "smem-cta"), (54, "l2-slot"),
                                      (18, "l2-slot"), (2, "l2-slot")])
def test_forced_regimes_match_zhegv(cuda, monkeypatch, n, regime):
    """Every kernel stays correct where the default choice no longer uses it
    (SUNNY_GENEIG_REGIME forces the regime at create time)."""
    from sunny_gen_eigensolver_b200 import Solver
    monkeypatch.setenv("SUNNY_GENEIG_REGIME", regime)
    with Solver(n) as s:
        assert s.regime == regime
        H, S = generators.baseline_problems(n, 5, seed=300 + n)
        W, U, info = gpu_solve(H, S, solver=s)
        check_against_zhegv(H, S, W, U, info)


def test_create_config_explicit_and_rejected(cuda):
    from sunny_gen_eigensolver_b200 import Solver
    with Solver(54, regime="l2-slot", slots_per_sm=1) as s:
        assert s.regime == "l2-slot"
        H, S = generators.baseline_problems(54, 3, seed=12)
        W, U, info = gpu_solve(H, S, solver=s)
        check_against_zhegv(H, S, W, U, info)
    for kw, msg in (({"regime": "smem-cta"}, "cannot hold"), ({"regime": "bogus"}, "unknown regime"),
                    ({"slots_per_sm": 3}, "slots_per_sm")):
        with pytest.raises(RuntimeError, match=msg):
            Solver(100, **kw)


def test_graph_replay_ordered_with_launches_on_other_streams(cuda):
    """An l2-slot handle (scratch slots shared by all its launches) used both
    by a captured CUDA graph replayed on one stream and by normal launches on
    another stream, with the replays ordered against the launches by the
    caller as the header asks: every result equals the one-at-a-time result
    bit for bit, and the capture does not disturb the handle."""
    import torch
    from sunny_gen_eigensolver_b200 import Solver, to_colmajor
    n, batch = 72, 96
    HA, SA = generators.baseline_problems(n, batch, seed=71)
    HB, SB = generators.baseline_problems(n, batch, seed=72)
    dev = torch.device("cuda")
    bufs = []
    for H, S in ((HA, SA), (HB, SB)):
        bufs.append((to_colmajor(torch.from_numpy(H).to(dev)), to_colmajor(torch.from_numpy(S).to(dev)),
                     torch.zeros((batch, n), dtype=torch.float64, device=dev),
                     torch.zeros((batch, n, n), dtype=torch.complex128, device=dev),
                     torch.zeros((batch,), dtype=torch.int32, device=dev)))
    with Solver(n) as s:
        assert s.regime == "l2-slot"
        ref = []
        for Hc, Sc, W, U, info in bufs:
            s.launch(Hc, Sc, W, U, info)
            torch.cuda.synchronize()
            ref.append((W.clone(), U.clone(), info.clone()))
            W.zero_(); U.zero_(); info.fill_(-7)
        s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        g = torch.cuda.CUDAGraph()
        s1.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.graph(g, stream=s1):
            s.launch(*bufs[0], stream=s1)
        for _ in range(3):
            with torch.cuda.stream(s1):
                g.replay()
            s2.wait_stream(s1)             # the caller orders replays against launches
            s.launch(*bufs[1], stream=s2)
            s.launch(*bufs[1], stream=s2)
            s1.wait_stream(s2)
        torch.cuda.synchronize()
        for (Hc, Sc, W, U, info), (Wr, Ur, ir) in zip(bufs, ref):
            assert torch.equal(info, ir) and torch.equal(W, Wr) and torch.equal(U, Ur)
        del g
