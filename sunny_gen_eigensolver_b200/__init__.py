"""B200-native (sm_100a) batched complex Hermitian-definite generalized
eigensolver H u = lambda S u, drop-in for the libsunny_geneig C ABI.

The solver itself is the compiled library lib/libsunny_geneig.so (CUDA
kernels + C ABI, include/sunny_geneig.h); this package holds its host-side
binding (`Solver`, mirroring the reference's Julia wrapper), the input
generators used by the benchmark and the accuracy measures.
"""
from .solver import Solver, UnevenSolver, from_colmajor, last_error, solve, to_colmajor  # noqa: F401

__all__ = ["Solver", "UnevenSolver", "solve", "to_colmajor", "from_colmajor", "last_error"]
