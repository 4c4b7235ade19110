"""sunny_geneig_launch_noalloc: the solve for callers that cannot allocate
device memory (code inside another framework's memory pool or under a
no-allocation policy, plugins whose host forbids cudaMalloc, graph-replay
setups that must not touch the allocator). It takes no handle; up to n = 60
it runs the shared-memory kernel, which needs no scratch, and above that it
uses a fixed device array built into the library as its scratch (n = 54 and
n = 96 below cover both).

Checked here through the C ABI against the regular entry point
(sunny_geneig_create_ex + sunny_geneig_launch) on the same inputs, on two
calls in a row, with the parity tolerances the other GPU tests use:
eigenvalues within 1e-12 ||H||_2, eigenvectors by S-inner-product phase
(1 - |u^H S u_ref| < 1e-10 where the eigenvalue gap is >= 1e-6), identical
info codes. This file is collected last so that a run stopping at the
first failure has run every other test before it.
"""
import numpy as np
import pytest

from sunny_gen_eigensolver_b200 import accuracy, generators

pytestmark = pytest.mark.gpu


def _buffers(torch, H, S):
    from sunny_gen_eigensolver_b200 import to_colmajor
    batch, n, _ = H.shape
    Hc = to_colmajor(torch.from_numpy(H).cuda())
    Sc = to_colmajor(torch.from_numpy(S).cuda())
    W = torch.full((batch, n), 7.0, dtype=torch.float64, device="cuda")
    U = torch.full((batch, n, n), 7.0 + 7.0j, dtype=torch.complex128, device="cuda")
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    return Hc, Sc, W, U, info


@pytest.mark.parametrize("n", [54, 96])
def test_noalloc_matches_regular_entry_point_twice(cuda, n):
    import torch
    from sunny_gen_eigensolver_b200 import Solver, _native as nat
    L = nat.load()
    H, S = generators.baseline_problems(n, 9, seed=4242 + n)
    S[4] = np.eye(n)
    S[4, 5, 5] = -2.0                      # one matrix with a non-PD S: info = n + 6
    Hc, Sc, Wr, Ur, ir = _buffers(torch, H, S)
    with Solver(n) as s:
        s.launch(Hc, Sc, Wr, Ur, ir)
    torch.cuda.synchronize()
    Wr, Ur, ir = Wr.cpu().numpy(), Ur.transpose(-1, -2).cpu().numpy(), ir.cpu().numpy()
    assert ir[4] == n + 6 and (np.delete(ir, 4) == 0).all()
    ok = ir == 0
    for call in range(2):
        _, _, W, U, info = _buffers(torch, H, S)
        st = L.sunny_geneig_launch_noalloc(n, Hc.data_ptr(), Sc.data_ptr(), W.data_ptr(), U.data_ptr(),
                                           info.data_ptr(), H.shape[0], torch.cuda.current_stream().cuda_stream)
        assert st == nat.STATUS_OK, nat.last_error()
        torch.cuda.synchronize()
        W, U, info = W.cpu().numpy(), U.transpose(-1, -2).cpu().numpy(), info.cpu().numpy()
        assert np.array_equal(info, ir), (call, info, ir)
        assert np.isnan(W[4]).all() and np.isnan(U[4]).all()
        assert accuracy.eig_err_rel(H[ok], W[ok], Wr[ok]).max() <= 1e-12
        assert accuracy.phase_err(S[ok], U[ok], Ur[ok], Wr[ok]).max() < 1e-10
        assert accuracy.residual(H[ok], S[ok], W[ok], U[ok]).max() <= 1e-12
        assert accuracy.s_orth(S[ok], U[ok]).max() <= 1e-12


def test_noalloc_rejects_bad_arguments(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import _native as nat
    L = nat.load()
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert L.sunny_geneig_launch_noalloc(513, p, p, p, p, p, 1, 0) == nat.STATUS_INVALID_ARG
    assert "outside" in nat.last_error()
    assert L.sunny_geneig_launch_noalloc(0, p, p, p, p, p, 1, 0) == nat.STATUS_INVALID_ARG
    assert L.sunny_geneig_launch_noalloc(8, p, p, p, p, p, -1, 0) == nat.STATUS_INVALID_ARG
    assert L.sunny_geneig_launch_noalloc(8, 0, p, p, p, p, 1, 0) == nat.STATUS_INVALID_ARG
    assert L.sunny_geneig_launch_noalloc(8, p + 8, p, p, p, p, 1, 0) == nat.STATUS_INVALID_ARG
    assert L.sunny_geneig_launch_noalloc(8, p, p, p, p, p, 0, 0) == nat.STATUS_OK
