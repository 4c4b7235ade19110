"""Continuous-batching serving loop for dispersion requests.

A request is one q-path or powder shell of a spin-wave calculation: `q`
matrix pairs (H, S) of one size N, solved together. Requests arrive over
time (Poisson in the benchmark); the engine

* admits waiting requests first-come-first-served whenever a stream slot
  and enough of the device-memory budget are free (a request needs
  q * (48 N^2 + 8 N + 4) bytes for H, S, U, W and info),
* starts each admitted request at once on its own stream, so requests that
  arrive while others are on the GPU overlap with them on the device,
* keeps inputs and results on the device (the client reads W / U from the
  finished request's tensors, or never: Sunny's intensity step consumes them
  on the device),
* releases a request's budget as soon as its completion event fires and
  admits the next ones,
* survives a failed start (the executor could not allocate the request's
  buffers): the request goes back to the head of the queue, the engine
  admits nothing more until an in-flight request has finished and freed
  memory, then retries; a request that cannot start even with nothing else
  in flight fails with the error as its result,
* records per-request latency (arrival to completion) and reports p50/p99
  latency, solves/s and queue statistics.

The GPU work goes through an executor (`DeviceExecutor`: per N a small pool
of Solver handles, so that requests of the same N can overlap on the device,
in the plain FP64 or the mixed-precision form, a pool of CUDA streams, the C
ABI launch); `SimExecutor` replaces it with a clock model so that the
admission logic can be tested without a GPU.
"""
from __future__ import annotations

import heapq
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np


def request_bytes(n: int, q: int) -> int:
    """Device bytes a request holds while admitted: H, S, U (complex128),
    W (float64) and info (int32) for q matrices of size n."""
    return q * (48 * n * n + 8 * n + 4)


@dataclass
class Request:
    rid: int
    n: int
    q: int
    arrival: float                 # seconds after the start of the run
    seed: int = 0
    # filled by the engine
    admitted: float = math.nan
    done: float = math.nan
    result: object = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeStats:
    completed: int = 0
    solves: int = 0
    wall_s: float = 0.0
    p50_ms: float = math.nan
    p99_ms: float = math.nan
    max_ms: float = math.nan
    mean_queue_wait_ms: float = math.nan
    max_waiting: int = 0
    max_in_flight: int = 0
    peak_budget_bytes: int = 0
    start_failures: int = 0        # starts the executor could not allocate (retried)
    failed_requests: int = 0       # requests that could not start at all
    by_n: Dict[int, int] = field(default_factory=dict)

    @property
    def solves_per_s(self) -> float:
        return self.solves / self.wall_s if self.wall_s > 0 else math.nan

    def as_dict(self):
        d = dict(self.__dict__)
        d["solves_per_s"] = self.solves_per_s
        return d


def poisson_requests(rate_hz: float, duration_s: float, sizes, q_range=(64, 4096), seed: int = 0,
                     size_weights=None) -> List[Request]:
    """Poisson arrivals at `rate_hz` over `duration_s`; N drawn from `sizes`
    (optionally weighted), q log-uniform on q_range."""
    rng = np.random.default_rng(seed)
    reqs, t, rid = [], 0.0, 0
    lo, hi = math.log(q_range[0]), math.log(q_range[1])
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        n = int(rng.choice(sizes, p=size_weights))
        q = int(round(math.exp(rng.uniform(lo, hi))))
        reqs.append(Request(rid=rid, n=n, q=q, arrival=t, seed=int(rng.integers(1 << 31))))
        rid += 1
    return reqs


class ServingEngine:
    """FIFO admission by slot and device-memory budget; see module docstring."""

    def __init__(self, executor, budget_bytes: int = 150 * 10 ** 9, max_in_flight: Optional[int] = None,
                 consume=None):
        """`consume(request, result)`, when given, receives each finished
        request's result (W, U, info on the device) at completion, like a
        client reading its answer, and the engine keeps nothing of it;
        otherwise the result stays on the request (`Request.result`)."""
        self.ex = executor
        self.budget = int(budget_bytes)
        self.slots = max_in_flight or executor.slots
        self.consume = consume

    def run(self, requests: List[Request], realtime: bool = True) -> ServeStats:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in pending:
            if request_bytes(r.n, r.q) > self.budget:
                raise ValueError(f"request {r.rid} needs more than the whole budget")
        waiting: List[Request] = []
        in_flight: List[tuple] = []          # (request, handle)
        used = 0
        blocked = 0                          # in-flight count at a failed start (0: admitting)
        st = ServeStats()
        clock = self.ex.clock
        t0 = clock()
        i = 0
        while i < len(pending) or waiting or in_flight:
            now = clock() - t0
            while i < len(pending) and (pending[i].arrival <= now or not realtime):
                waiting.append(pending[i])
                i += 1
            st.max_waiting = max(st.max_waiting, len(waiting))
            # retire finished requests, freeing their budget and slot
            still = []
            for r, h in in_flight:
                if self.ex.finished(h):
                    r.done = clock() - t0
                    res = self.ex.result(h)
                    if self.consume is not None:
                        self.consume(r, res)
                    else:
                        r.result = res
                    used -= request_bytes(r.n, r.q)
                    st.completed += 1
                    st.solves += r.q
                    st.by_n[r.n] = st.by_n.get(r.n, 0) + r.q
                else:
                    still.append((r, h))
            in_flight = still
            # admit in arrival order while a slot and the budget allow; after a
            # failed start admit nothing until an in-flight request finishes
            if blocked and len(in_flight) < blocked:
                blocked = 0
            while waiting and len(in_flight) < self.slots and not blocked:
                r = waiting[0]
                need = request_bytes(r.n, r.q)
                if used + need > self.budget:
                    break
                try:
                    h = self.ex.start(r)
                except (MemoryError, RuntimeError) as err:
                    st.start_failures += 1
                    if in_flight:
                        blocked = len(in_flight)      # retry once one of these has finished
                        break
                    waiting.pop(0)                    # nothing else holds memory: give up on it
                    r.admitted = r.done = clock() - t0
                    st.failed_requests += 1
                    if self.consume is not None:
                        self.consume(r, err)
                    else:
                        r.result = err
                    continue
                waiting.pop(0)
                used += need
                r.admitted = clock() - t0
                in_flight.append((r, h))
                st.peak_budget_bytes = max(st.peak_budget_bytes, used)
            st.max_in_flight = max(st.max_in_flight, len(in_flight))
            next_arrival = t0 + pending[i].arrival if (i < len(pending) and realtime) else None
            self.ex.wait(next_arrival, busy=bool(in_flight))
        st.wall_s = clock() - t0
        lat = np.array([r.latency for r in requests]) * 1e3
        waits = np.array([r.admitted - r.arrival for r in requests]) * 1e3
        if len(lat):
            st.p50_ms, st.p99_ms, st.max_ms = (float(np.percentile(lat, 50)), float(np.percentile(lat, 99)),
                                               float(lat.max()))
            st.mean_queue_wait_ms = float(waits.mean())
        return st


class SimExecutor:
    """Clock model of the device for CPU tests: each request takes
    q / rate[n] seconds on one of `slots` independent lanes, in simulated time."""

    def __init__(self, rate: Dict[int, float], slots: int = 4):
        self.rate, self.slots = rate, slots
        self.now = 0.0
        self._busy = []          # heap of finish times

    def clock(self):
        return self.now

    def start(self, r: Request):
        fin = self.now + r.q / self.rate[r.n]
        heapq.heappush(self._busy, fin)
        return {"finish": fin, "rid": r.rid}

    def finished(self, h):
        return h["finish"] <= self.now + 1e-12

    def result(self, h):
        return h["rid"]

    def wait(self, next_arrival, busy):
        # advance simulated time to the next completion or arrival
        while self._busy and self._busy[0] <= self.now:
            heapq.heappop(self._busy)
        cand = [t for t in ((self._busy[0] if self._busy else None), next_arrival) if t is not None]
        self.now = max(self.now, min(cand)) if cand else self.now


class DeviceExecutor:
    """Runs requests on one GPU through the C ABI: one Solver per N, a pool
    of CUDA streams, inputs drawn on the device from a per-N pool of seeded
    problems (a stand-in for Sunny's on-device assembly of H and S)."""

    def __init__(self, device: int = 0, slots: int = 8, pool_size: int = 256, kappa: float = 100.0,
                 poll_sleep_s: float = 50e-6, kernel: str = "unified", handles_per_n: int = 2):
        """`kernel`: "unified" (plain FP64) or "mixed" (FP32 reduction + FP64
        refinement). `handles_per_n`: Solver handles per size; a handle whose
        solver keeps scratch slots serialises its own launches, so two
        handles let two requests of one N run on the device at once."""
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.slots = slots
        self.pool_size, self.kappa = pool_size, kappa
        self.kernel = kernel
        self.handles_per_n = max(1, int(handles_per_n))
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(slots)]
        self._next_stream = 0
        self.solvers: Dict[int, object] = {}          # first handle per N (regime queries)
        self.handles: Dict[int, list] = {}            # N -> [[solver, requests in flight], ...]
        self.pools: Dict[int, tuple] = {}
        self.poll_sleep_s = poll_sleep_s

    def clock(self):
        return time.perf_counter()

    def prepare(self, sizes):
        """Create the per-N solvers and input pools up front (outside the timed run)."""
        from .generators import baseline_problems_torch
        from .solver import Solver
        for n in sorted(set(sizes)):
            if n in self.solvers:
                continue
            first = Solver(n, device_id=self.dev.index or 0, kernel=self.kernel)
            self.solvers[n] = first
            # smem-cta solvers keep no scratch: one handle serves any overlap
            count = 1 if first.regime == "smem-cta" else self.handles_per_n
            self.handles[n] = [[first, 0]] + [[Solver(n, device_id=self.dev.index or 0, kernel=self.kernel), 0]
                                              for _ in range(count - 1)]
            H, S = baseline_problems_torch(n, self.pool_size, seed=777 + n, kappa=self.kappa, device=self.dev)
            self.pools[n] = (H.transpose(-1, -2).contiguous(), S.transpose(-1, -2).contiguous())
        self.torch.cuda.synchronize(self.dev)

    def inputs(self, r: Request):
        """The request's q input pairs (column-major buffers), drawn from the pool by its seed."""
        torch = self.torch
        Hp, Sp = self.pools[r.n]
        g = torch.Generator(device="cpu")
        g.manual_seed(r.seed)
        idx = torch.randint(0, Hp.shape[0], (r.q,), generator=g).to(self.dev)
        return Hp.index_select(0, idx), Sp.index_select(0, idx)

    def start(self, r: Request):
        torch = self.torch
        s = self.streams[self._next_stream]
        self._next_stream = (self._next_stream + 1) % len(self.streams)
        with torch.cuda.stream(s):
            H, S = self.inputs(r)
            W = torch.empty((r.q, r.n), dtype=torch.float64, device=self.dev)
            U = torch.empty((r.q, r.n, r.n), dtype=torch.complex128, device=self.dev)
            info = torch.empty((r.q,), dtype=torch.int32, device=self.dev)
            slot = min(self.handles[r.n], key=lambda hs: hs[1])    # the least busy handle of this N
            slot[0].launch(H, S, W, U, info, s)
            slot[1] += 1
            ev = torch.cuda.Event()
            ev.record(s)
        return {"event": ev, "out": (W, U, info), "keep": (H, S), "stream": s, "handle": slot}

    def finished(self, h):
        return h["event"].query()

    def result(self, h):
        h.pop("keep", None)
        slot = h.pop("handle", None)
        if slot is not None:
            slot[1] -= 1
        return h["out"]

    def close(self):
        for hs in self.handles.values():
            for solver, _ in hs:
                solver.close()
        self.handles.clear()
        self.solvers.clear()

    def wait(self, next_arrival, busy):
        if busy or next_arrival is None:
            time.sleep(self.poll_sleep_s)
        else:
            time.sleep(max(0.0, min(next_arrival - time.perf_counter(), 0.01)))
