"""Linear spin-wave dynamical matrices as Fourier terms for the fused
assembly entry points (sunny_geneig_launch_fourier_sigma[_intensity]).

The reference's caller builds the metric-side matrix with Sunny's
`dynamical_matrix!` on the host or GPU and passes it to the solver
(julia/SunnyGeneigBench/scripts/setup_sw08.jl:103, called before the
solve at :54-76). Sunny's code is not part of the reference, so this module
restates the published linear spin-wave construction (Holstein-Primakoff
to quadratic order in the local frame of each ordered moment, as in
S. Toth and B. Lake, J. Phys.: Condens. Matter 27, 166002 (2015)) for
bilinear exchange between sites and Zeeman fields.

Model: m sites per magnetic cell with spin lengths S_a and ordered
directions n_a; bonds (a, b, d, J): S_a(r)^T J S_b(r + d) summed over cells
r, each bond listed once (d in lattice units, J a real 3x3 matrix); fields
h_a: -h_a . S_a. With u_a = e1 + i e2 of a right-handed frame (e1, e2, n_a),
the quadratic Hamiltonian is (1/2) sum_q x^dag h(q) x with
x = (a(q), a(-q)^dag) and

    h(q) = [[M(q), P(q)], [P(q)^dag, conj(M(-q))]],
    M_ab(q) += c1 e^{i k.d},  M_ba(q) += conj(c1) e^{-i k.d},
    P_ab(q) += c2 e^{i k.d},  P_ba(q) += c2 e^{-i k.d},
    c1 = sqrt(S_a S_b)/2 u_a^T J conj(u_b),  c2 = sqrt(S_a S_b)/2 u_a^T J u_b,
    M_aa += -(n_a^T J n_b) S_b,  M_bb += -(n_a^T J n_b) S_a,  M_aa += h_a . n_a,

k = 2 pi q (q in reciprocal-lattice units). The magnon energies are the
positive eigenvalues of diag(I, -I) h(q): the solver's metric form
H u = lambda S u with H = diag(I, -I) and S = h(q) gives omega = 1 / lambda
for lambda > 0. h(q) must be positive definite (a stable ordered state with
gapped modes), as for Sunny's metric solve.

Pinned by the analytic dispersions of the Heisenberg ferromagnetic chain in
a field, omega = 2|J|S(1 - cos k) + h, and of the antiferromagnetic chain in a
staggered field, omega = sqrt((2JS + h)^2 - (2JS cos(k/2))^2) (two-site
cell), in tests/test_lswt.py.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np


def local_frame(n: Sequence[float]) -> Tuple[np.ndarray, np.ndarray]:
    """(u, n): u = e1 + i e2 for a right-handed orthonormal frame (e1, e2, n)."""
    n = np.asarray(n, dtype=np.float64)
    n = n / np.linalg.norm(n)
    a = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(a, n)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(n, e1)
    return e1 + 1j * e2, n


@dataclass
class SpinModel:
    """Ordered magnetic cell: spins[a] = S_a, directions[a] = n_a (any
    length), bonds (a, b, d, J) each listed once, fields[a] = h_a."""
    spins: List[float]
    directions: List[Sequence[float]]
    bonds: List[Tuple[int, int, Sequence[float], np.ndarray]] = field(default_factory=list)
    fields: List[Sequence[float]] = field(default_factory=list)

    @property
    def m(self) -> int:
        return len(self.spins)

    @property
    def n(self) -> int:
        return 2 * len(self.spins)


def fourier_terms(model: SpinModel):
    """Terms (rows, cols, coef, disp) of h(q): entry (rows[t], cols[t]) gets
    coef[t] exp(2 pi i q . disp[t]). All entries (both triangles)."""
    m = model.m
    frames = [local_frame(d) for d in model.directions]
    rows, cols, coef, disp = [], [], [], []

    def add(r, c, v, d):
        rows.append(r); cols.append(c); coef.append(complex(v)); disp.append(np.asarray(d, dtype=np.float64))

    zero = np.zeros(3)
    for a, b, d, J in model.bonds:
        J = np.asarray(J, dtype=np.float64)
        d = np.asarray(d, dtype=np.float64)
        ua, na = frames[a]
        ub, nb = frames[b]
        s = np.sqrt(model.spins[a] * model.spins[b]) / 2.0
        c1 = s * (ua @ J @ ub.conj())
        c2 = s * (ua @ J @ ub)
        add(a, b, c1, d)                                  # M(q)
        add(b, a, np.conj(c1), -d)
        add(a, m + b, c2, d)                              # P(q)
        add(b, m + a, c2, -d)
        add(m + b, a, np.conj(c2), -d)                    # P(q)^dag
        add(m + a, b, np.conj(c2), d)
        add(m + a, m + b, np.conj(c1), d)                 # conj(M(-q))
        add(m + b, m + a, c1, -d)
        L = float(na @ J @ nb)
        for i, v in ((a, -L * model.spins[b]), (b, -L * model.spins[a])):
            add(i, i, v, zero)
            add(m + i, m + i, v, zero)
    for i, h in enumerate(model.fields):
        v = float(np.dot(h, frames[i][1]))
        add(i, i, v, zero)
        add(m + i, m + i, v, zero)
    return (np.asarray(rows, dtype=np.int64), np.asarray(cols, dtype=np.int64),
            np.asarray(coef, dtype=np.complex128), np.asarray(disp, dtype=np.float64).reshape(-1, 3))


def pack_terms(n: int, rows, cols, coef, disp, lower_only: bool = True):
    """Sorted term table of the device entry points: start int32[n*n + 1]
    (entry e = row + n col owns terms [start[e], start[e+1])), coef
    complex128[nt], disp float64[nt, 3]. lower_only keeps the row >= col
    entries, the only ones the device reads."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    if rows.size and (rows.min() < 0 or cols.min() < 0 or rows.max() >= n or cols.max() >= n):
        raise ValueError("term index outside the n x n matrix")
    keep = rows >= cols if lower_only else np.ones(rows.shape, dtype=bool)
    e = (rows + n * cols)[keep]
    order = np.argsort(e, kind="stable")
    e = e[order]
    start = np.zeros(n * n + 1, dtype=np.int64)
    np.add.at(start, e + 1, 1)
    start = np.cumsum(start)
    if start[-1] > np.iinfo(np.int32).max:
        raise ValueError("too many terms for int32 offsets")
    return (start.astype(np.int32), np.ascontiguousarray(np.asarray(coef)[keep][order], dtype=np.complex128),
            np.ascontiguousarray(np.asarray(disp)[keep][order], dtype=np.float64))


def random_model(m: int, n_bonds: int, seed: int, spin: float = 1.0, field_strength: float = 2.0) -> SpinModel:
    """A seeded ordered model that stays stable: ferromagnetic order along z,
    random ferromagnetic couplings with a small in-plane anisotropy on random
    bonds, and a uniform field along z that gaps every mode (the test and benchmark input
    of the fused assembly; its size mimics the 27-site SW08 cell at m = 27)."""
    rng = np.random.default_rng(seed)
    bonds = []
    for _ in range(n_bonds):
        a, b = (int(x) for x in rng.integers(0, m, size=2))
        d = rng.integers(-1, 2, size=3).astype(np.float64)
        if a == b and not d.any():
            d[0] = 1.0
        # symmetric in-plane anisotropy only (J z || z keeps the z order stationary)
        Jxy = rng.normal(size=(2, 2)) * 0.05
        J = -np.eye(3) * rng.uniform(0.2, 1.0)
        J[:2, :2] += 0.5 * (Jxy + Jxy.T)
        bonds.append((a, b, d, J))
    return SpinModel(spins=[spin] * m, directions=[[0.0, 0.0, 1.0]] * m, bonds=bonds,
                     fields=[[0.0, 0.0, field_strength]] * m)
