"""ORACLE (test infrastructure): the Fourier-sum assembly of the metric-side
matrix that the fused entry points (sunny_geneig_launch_fourier_sigma and
its intensity form) run on the device, restated with numpy.

For each problem b with wavevector q_b (reciprocal-lattice units) and a term
list (rows, cols, coef, disp):

    S(q_b)[rows[t], cols[t]] += coef[t] * exp(2 pi i q_b . disp[t]).

This is the step the reference's caller runs before the solve (Sunny's
`dynamical_matrix!`, julia/SunnyGeneigBench/scripts/setup_sw08.jl:103).
Sunny's code is not part of the reference, so parity with Sunny's own
matrices is unpinned; the spin-wave front end that produces the terms
(sunny_gen_eigensolver_b200.lswt) is pinned instead to the analytic
dispersions of the ferromagnetic and antiferromagnetic Heisenberg chains
(tests/test_lswt.py). Only tests and the benchmark's checks use this file.
"""
import numpy as np


def assemble(n, rows, cols, coef, disp, q):
    """(batch, n, n) complex128 matrices (natural layout) for q of shape
    (batch, 3); every term is applied (both triangles, as given)."""
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3)
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    coef = np.asarray(coef, dtype=np.complex128)
    disp = np.asarray(disp, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((q.shape[0], n, n), dtype=np.complex128)
    ph = np.exp(2j * np.pi * (q @ disp.T))              # (batch, nt)
    vals = ph * coef[None, :]
    for b in range(q.shape[0]):
        np.add.at(out[b], (rows, cols), vals[b])
    return out


def magnon_energies(S):
    """Positive eigenvalues of diag(I, -I) S per problem, ascending: the
    spin-wave energies of a dynamical matrix S (batch, n, n)."""
    S = np.asarray(S)
    n = S.shape[-1]
    m = n // 2
    g = np.concatenate([np.ones(m), -np.ones(m)])
    ev = np.linalg.eigvals(g[None, :, None] * S)
    ev = np.sort(ev.real, axis=-1)
    return ev[:, m:]
