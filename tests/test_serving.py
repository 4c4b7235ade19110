"""Serving loop: admission and accounting on a clock model (CPU), and on the
GPU the property that every request's result is the same alone and in the mix."""
import math

import numpy as np
import pytest

from sunny_gen_eigensolver_b200.serving import (Request, ServingEngine, SimExecutor, poisson_requests,
                                                request_bytes)


def test_request_bytes():
    assert request_bytes(54, 1) == 48 * 54 * 54 + 8 * 54 + 4


def test_fifo_single_slot_latencies():
    ex = SimExecutor({8: 100.0}, slots=1)            # 100 solves/s
    reqs = [Request(rid=k, n=8, q=10, arrival=0.0) for k in range(3)]
    st = ServingEngine(ex, budget_bytes=10 ** 12).run(reqs)
    assert [round(r.done, 6) for r in reqs] == [0.1, 0.2, 0.3]
    assert st.completed == 3 and st.solves == 30 and math.isclose(st.solves_per_s, 100.0)
    assert st.max_in_flight == 1 and st.max_waiting == 3


def test_budget_limits_concurrency_and_frees_on_completion():
    ex = SimExecutor({8: 100.0}, slots=8)
    one = request_bytes(8, 10)
    reqs = [Request(rid=k, n=8, q=10, arrival=0.0) for k in range(4)]
    st = ServingEngine(ex, budget_bytes=2 * one).run(reqs)
    assert st.max_in_flight == 2 and st.peak_budget_bytes == 2 * one
    assert sorted(round(r.done, 6) for r in reqs) == [0.1, 0.1, 0.2, 0.2]


def test_late_arrivals_are_admitted_while_others_run():
    ex = SimExecutor({8: 10.0, 16: 10.0}, slots=4)
    reqs = [Request(rid=0, n=8, q=20, arrival=0.0), Request(rid=1, n=16, q=1, arrival=0.5)]
    ServingEngine(ex, budget_bytes=10 ** 12).run(reqs)
    assert math.isclose(reqs[1].admitted, 0.5) and math.isclose(reqs[1].done, 0.6)
    assert math.isclose(reqs[0].done, 2.0)


def test_oversized_request_rejected():
    ex = SimExecutor({8: 10.0})
    with pytest.raises(ValueError):
        ServingEngine(ex, budget_bytes=10).run([Request(rid=0, n=8, q=1, arrival=0.0)])


def test_poisson_generator():
    reqs = poisson_requests(200.0, 2.0, [18, 54], seed=3)
    assert 300 < len(reqs) < 500
    assert all(64 <= r.q <= 4096 and r.n in (18, 54) for r in reqs)
    assert all(a.arrival < b.arrival for a, b in zip(reqs, reqs[1:]))


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix(cuda):
    import torch
    from sunny_gen_eigensolver_b200.serving import DeviceExecutor
    sizes = [18, 54, 108]
    reqs = poisson_requests(400.0, 0.05, sizes, q_range=(16, 96), seed=11)
    assert len(reqs) >= 6
    ex = DeviceExecutor(slots=4, pool_size=64)
    ex.prepare(sizes)
    ServingEngine(ex, budget_bytes=4 * 10 ** 9).run(reqs)
    torch.cuda.synchronize()
    for r in reqs:
        W, U, info = r.result
        alone = Request(rid=r.rid, n=r.n, q=r.q, arrival=0.0, seed=r.seed)
        ServingEngine(ex, budget_bytes=4 * 10 ** 9, max_in_flight=1).run([alone])
        torch.cuda.synchronize()
        W1, U1, i1 = alone.result
        assert torch.equal(info, i1) and bool((info == 0).all())
        assert torch.equal(W, W1) and torch.equal(U, U1)


def test_consumer_receives_every_result_once_and_nothing_is_kept():
    reqs = poisson_requests(200.0, 0.5, [18, 54], q_range=(64, 256), seed=3)
    got = []
    eng = ServingEngine(SimExecutor({18: 1e6, 54: 2e5}, slots=4), budget_bytes=10 ** 9,
                        consume=lambda r, res: got.append((r.rid, res)))
    st = eng.run(reqs)
    assert st.completed == len(reqs) and sorted(rid for rid, _ in got) == sorted(r.rid for r in reqs)
    assert all(res == rid for rid, res in got)          # SimExecutor's result is the request id
    assert all(r.result is None for r in reqs)


class _FailingSim(SimExecutor):
    """SimExecutor whose start() fails with an allocation error for the
    request ids in `fail_ids`, `times` times each (host-side fault injection:
    the stand-in for a cudaMalloc / torch allocation that runs out of memory)."""

    def __init__(self, rate, slots, fail_ids, times=1):
        super().__init__(rate, slots)
        self.left = {rid: times for rid in fail_ids}

    def start(self, r):
        if self.left.get(r.rid, 0) > 0:
            self.left[r.rid] -= 1
            raise MemoryError(f"injected allocation failure for request {r.rid}")
        return super().start(r)


def test_failed_start_is_retried_after_memory_frees():
    ex = _FailingSim({8: 100.0}, slots=4, fail_ids=[1])
    reqs = [Request(rid=0, n=8, q=10, arrival=0.0), Request(rid=1, n=8, q=10, arrival=0.0),
            Request(rid=2, n=8, q=10, arrival=0.0)]
    st = ServingEngine(ex, budget_bytes=10 ** 12).run(reqs)
    assert st.start_failures == 1 and st.failed_requests == 0 and st.completed == 3
    # request 1 waits for request 0 to finish (0.1 s), then starts; 2 stays behind it (FIFO)
    assert math.isclose(reqs[0].done, 0.1) and math.isclose(reqs[1].admitted, 0.1)
    assert math.isclose(reqs[1].done, 0.2) and math.isclose(reqs[2].admitted, 0.1)
    assert reqs[1].result == 1


def test_request_that_never_starts_fails_without_blocking_the_queue():
    ex = _FailingSim({8: 100.0}, slots=2, fail_ids=[0], times=10 ** 6)
    reqs = [Request(rid=0, n=8, q=10, arrival=0.0), Request(rid=1, n=8, q=10, arrival=0.05)]
    st = ServingEngine(ex, budget_bytes=10 ** 12).run(reqs)
    assert st.failed_requests == 1 and st.completed == 1
    assert isinstance(reqs[0].result, MemoryError)
    assert math.isclose(reqs[1].done, 0.15)


@pytest.mark.gpu
def test_mixed_form_serving_matches_plain_within_tolerance(cuda):
    import torch
    from sunny_gen_eigensolver_b200.serving import DeviceExecutor
    sizes = [18, 54]
    reqs = poisson_requests(400.0, 0.03, sizes, q_range=(16, 64), seed=5)
    out = {}
    for kernel in ("unified", "mixed"):
        ex = DeviceExecutor(slots=4, pool_size=32, kernel=kernel)
        ex.prepare(sizes)
        copies = [Request(rid=r.rid, n=r.n, q=r.q, arrival=r.arrival, seed=r.seed) for r in reqs]
        ServingEngine(ex, budget_bytes=2 * 10 ** 9).run(copies)
        torch.cuda.synchronize()
        out[kernel] = {r.rid: r.result for r in copies}
        ex.close()
    for rid, (Wp, _, ip) in out["unified"].items():
        Wm, _, im = out["mixed"][rid]
        assert torch.equal(ip, im) and bool((ip == 0).all())
        scale = Wp.abs().amax(dim=1)
        assert float(((Wm - Wp).abs().amax(dim=1) / scale).max()) <= 1e-12
