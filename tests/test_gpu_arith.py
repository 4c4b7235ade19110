"""Device arithmetic the solver depends on, checked against CUDA's own
correctly rounded operations on the GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fast_reciprocal_within_one_ulp(cuda):
    import torch
    from sunny_gen_eigensolver_b200 import _native as nat
    L = nat.load()
    rng = np.random.default_rng(0)
    mant = rng.uniform(1.0, 2.0, 1 << 20)
    expo = rng.integers(-900, 900, 1 << 20)
    sign = rng.choice([-1.0, 1.0], 1 << 20)
    x = torch.from_numpy(sign * np.ldexp(mant, expo)).cuda()
    out = torch.empty_like(x)
    assert L.sunny_geneig_selftest_reciprocal(x.data_ptr(), out.data_ptr(), x.numel(), 0) == nat.STATUS_OK
    ref = 1.0 / x                     # CUDA IEEE division
    torch.cuda.synchronize()
    ulp = torch.abs(ref - out) / torch.abs(torch.nextafter(ref, torch.full_like(ref, float("inf"))) - ref)
    assert float(ulp.max()) <= 1.0
    assert float((ulp == 0).double().mean()) > 0.9
