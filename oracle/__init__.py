"""ORACLE -- test infrastructure, not part of the product.

CPU restatements of the reference's generalized eigensolve path
(src/unified/kernel_source.hpp:244-253: potrf -> trsm -> trsm -> heev ->
trsm) and of its LAPACK ground truth (LAPACKE_zhegv / zhegvd as used by
tests/common/lapack_reference.cpp:186-194 and tests/static/*), plus a
bit-exact restatement of the reference's seeded fixture generator
(fixture_gen.cpp) and a reader for its GEIG v1 fixture format.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker or the timed CPU baseline:
the solver's product path (libsunny_geneig.so) never calls into it.

Parity pinning: the restatements are checked against the reference's
golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
reference's tests/data/*.bin): the generator reproduces every fixture's H
and S bit-for-bit, and LAPACK zhegv reproduces the fixtures' eigenvalues to
~1e-15 relative.
"""
from .lapack import (  # noqa: F401
    zhegv_batch, zpotrf_batch, reduce_batch, zheev_batch, chain_batch,
)
