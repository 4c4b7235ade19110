"""Uneven-size batches: many problems whose N varies, solved by one graph launch.

Problems are grouped by N into packed, batch-contiguous buffers (one group
per size, the C-ABI layout). Each size class gets its own solver handle and
its own CUDA stream; all classes are launched concurrently and the whole set
of launches is captured once into a CUDA graph, so that a batch of the same
shape is re-run by a single graph launch (`UnevenBatch.replay`). The plain
alternative (`run_sequential`) is one launch per size on one stream.

The persistent form (`persistent` / `replay_persistent`) solves the whole mix
with ONE kernel launch (sunny_geneig_uneven_*): a device work counter hands
out items, largest N first, to a grid of 2 CTAs per SM, and each item runs
the per-problem code of its size's regime (results are bitwise those of
the per-size launches). `autotune_persistent` picks, per size, the regime
(smem-cta or l2-slot where both can hold N) and the problems per work item
(for smem-cta sizes) by timing the one-launch form on the batch's own data,
one size at a time from the library defaults; the choice is remembered per
size mix in the same table, and the launch is captured into a CUDA graph.

`autotune` picks, per size class, the execution configuration (which kernel
regime and, for the l2-slot kernel, how many CTAs per SM: `size_configs`)
by timing every candidate that can hold that N on the class's own data, and
then the launch plan (how many streams, which sizes share a stream, in which
order): it spreads the classes over k streams by longest-processing-time-
first for each candidate k, captures and times each candidate graph, and
keeps the fastest. Choices are remembered per size mix in an on-disk table
(`TuneTable`), written atomically (temporary file + rename) and validated
when read; a corrupt or foreign file is ignored and rewritten.
"""
from __future__ import annotations

import json
import os
import tempfile
from dataclasses import dataclass
from pathlib import Path
from typing import Dict, List, Optional, Sequence

TABLE_VERSION = 3


def size_configs(n: int) -> List[dict]:
    """Execution configurations tried for size n (those that cannot hold n
    are rejected by the library at create time and skipped)."""
    cands = [{"regime": "l2-slot", "slots_per_sm": 2}, {"regime": "l2-slot", "slots_per_sm": 1}]
    if n <= 64:
        cands.insert(0, {"regime": "smem-cta", "slots_per_sm": 0})
    elif n <= 96:
        cands.append({"regime": "smem-wide", "slots_per_sm": 0})
    return cands


def default_table_path() -> Path:
    env = os.environ.get("SUNNY_GENEIG_TUNE_TABLE")
    if env:
        return Path(env)
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(base) / "sunny_geneig" / "uneven_plans.json"


def mix_key(counts: Dict[int, int], device_name: str = "") -> str:
    """Key of a size mix: sizes with counts rounded to 2 significant figures."""
    def r2(c):
        s = f"{c:.2g}"
        return str(int(float(s)))
    return device_name + "|" + ",".join(f"{n}:{r2(c)}" for n, c in sorted(counts.items()))


@dataclass
class Plan:
    streams: List[List[int]]      # sizes launched on each stream, in order
    configs: Dict[int, dict] = None   # size -> {"regime": str, "slots_per_sm": int}
    # persistent form: size -> {"regime": "smem-cta" | "l2-slot", "per_item": int}
    persistent: Dict[int, dict] = None

    def to_json(self):
        return {"streams": self.streams, "configs": {str(n): c for n, c in (self.configs or {}).items()},
                "persistent": {str(n): c for n, c in (self.persistent or {}).items()}}

    @staticmethod
    def from_json(d) -> "Plan":
        if not isinstance(d, dict) or not isinstance(d.get("streams"), list):
            raise ValueError("bad plan")
        pers = {}
        for k, c in (d.get("persistent") or {}).items():
            if (not isinstance(c, dict) or c.get("regime") not in ("smem-cta", "l2-slot")
                    or not isinstance(c.get("per_item"), int) or not 1 <= c["per_item"] <= 64):
                raise ValueError("bad persistent config")
            pers[int(k)] = {"regime": c["regime"], "per_item": c["per_item"]}
        st = []
        for lane in d["streams"]:
            if not isinstance(lane, list) or not all(isinstance(x, int) and x > 0 for x in lane):
                raise ValueError("bad plan lane")
            st.append(list(lane))
        if not st:
            raise ValueError("empty plan")
        cfg = {}
        for k, c in (d.get("configs") or {}).items():
            if (not isinstance(c, dict) or c.get("regime") not in ("smem-cta", "smem-wide", "l2-slot")
                    or c.get("slots_per_sm") not in (0, 1, 2)):
                raise ValueError("bad size config")
            cfg[int(k)] = {"regime": c["regime"], "slots_per_sm": c["slots_per_sm"]}
        return Plan(st, cfg, pers)


class TuneTable:
    """Persisted {size mix -> Plan}; atomic writes, validated reads."""

    def __init__(self, path: Optional[Path] = None, enabled: bool = True):
        self.path = Path(path) if path else default_table_path()
        self.enabled = enabled
        self.plans: Dict[str, Plan] = {}
        self.rejected = False
        if enabled:
            self._load()

    def _load(self):
        try:
            raw = json.loads(self.path.read_text())
        except FileNotFoundError:
            return
        except (OSError, ValueError):
            self.rejected = True
            return
        try:
            if raw.get("format") != "sunny-geneig-uneven-plans" or raw.get("version") != TABLE_VERSION:
                raise ValueError("foreign table")
            self.plans = {str(k): Plan.from_json(v) for k, v in raw["plans"].items()}
        except (AttributeError, KeyError, TypeError, ValueError):
            self.plans = {}
            self.rejected = True

    def get(self, key: str) -> Optional[Plan]:
        return self.plans.get(key)

    def put(self, key: str, plan: Plan) -> None:
        self.plans[key] = plan
        if not self.enabled:
            return
        self.path.parent.mkdir(parents=True, exist_ok=True)
        body = {"format": "sunny-geneig-uneven-plans", "version": TABLE_VERSION,
                "plans": {k: p.to_json() for k, p in self.plans.items()}}
        fd, tmp = tempfile.mkstemp(prefix=".plans.", dir=str(self.path.parent))
        try:
            with os.fdopen(fd, "w") as f:
                json.dump(body, f)
            os.replace(tmp, self.path)
        except BaseException:
            try:
                os.unlink(tmp)
            except OSError:
                pass
            raise


def lpt_plan(cost: Dict[int, float], k: int) -> Plan:
    """Longest-processing-time-first assignment of size classes to k streams."""
    lanes = [[] for _ in range(max(1, min(k, len(cost))))]
    load = [0.0] * len(lanes)
    for n in sorted(cost, key=lambda x: -cost[x]):
        j = min(range(len(lanes)), key=lambda t: load[t])
        lanes[j].append(n)
        load[j] += cost[n]
    return Plan([l for l in lanes if l])


class UnevenBatch:
    """Device buffers and launches for a batch of problems of varying N.

    `sizes[p]` is the size of problem p; `set_inputs(n, H, S)` fills the
    column-major buffers of size class n (tensors of shape (count_n, n, n))."""

    def __init__(self, sizes: Sequence[int], device=None):
        import torch
        from .solver import Solver
        self.torch = torch
        self.dev = torch.device(device if device is not None else "cuda")
        counts: Dict[int, int] = {}
        for n in sizes:
            counts[int(n)] = counts.get(int(n), 0) + 1
        self.counts = dict(sorted(counts.items()))
        self.H, self.S, self.W, self.U, self.info = {}, {}, {}, {}, {}
        self.solvers, self.streams = {}, {}
        for n, c in self.counts.items():
            self.H[n] = torch.empty((c, n, n), dtype=torch.complex128, device=self.dev)
            self.S[n] = torch.empty((c, n, n), dtype=torch.complex128, device=self.dev)
            self.W[n] = torch.empty((c, n), dtype=torch.float64, device=self.dev)
            self.U[n] = torch.empty((c, n, n), dtype=torch.complex128, device=self.dev)
            self.info[n] = torch.empty((c,), dtype=torch.int32, device=self.dev)
            self.solvers[n] = Solver(n, device_id=self.dev.index or 0)
        self.graph = None
        self.plan: Optional[Plan] = None
        self.configs: Dict[int, dict] = {}
        self.uneven = None               # UnevenSolver of the persistent form
        self.pgraph = None               # its captured launch
        self.pconfigs: Dict[int, dict] = {}

    @property
    def total(self) -> int:
        return sum(self.counts.values())

    def set_inputs(self, n: int, H, S) -> None:
        self.H[n].copy_(H)
        self.S[n].copy_(S)

    def use_config(self, n: int, cfg: dict) -> None:
        """Replace size n's solver by one created with execution config `cfg`."""
        from .solver import Solver
        s = Solver(n, device_id=self.dev.index or 0, regime=cfg["regime"], slots_per_sm=cfg["slots_per_sm"])
        self.solvers[n].close()
        self.solvers[n] = s
        self.configs[n] = dict(cfg)
        self.graph = None

    def _launch(self, n, stream):
        self.solvers[n].launch(self.H[n], self.S[n], self.W[n], self.U[n], self.info[n], stream)

    def run_sequential(self, stream=None) -> None:
        """One plain launch per size class, one after the other on one stream."""
        s = stream or self.torch.cuda.current_stream(self.dev)
        for n in self.counts:
            self._launch(n, s)

    def _lane_streams(self, plan: Plan):
        torch = self.torch
        while len(self.streams) < len(plan.streams):
            self.streams[len(self.streams)] = torch.cuda.Stream(self.dev)
        return [self.streams[i] for i in range(len(plan.streams))]

    def capture(self, plan: Plan):
        """Capture the launches of `plan` into one CUDA graph (each size class on
        its plan stream: the same stream it is warmed up on, so that handles
        with scratch slots never wait across streams)."""
        torch = self.torch
        lanes = self._lane_streams(plan)
        cur = torch.cuda.current_stream(self.dev)
        for lane, s in zip(plan.streams, lanes):      # warm-up on the capture streams
            s.wait_stream(cur)
            for n in lane:
                self._launch(n, s)
            cur.wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        root = lanes[0]
        with torch.cuda.graph(g, stream=root):
            for lane, s in zip(plan.streams, lanes):
                if s is not root:
                    s.wait_stream(root)
                for n in lane:
                    self._launch(n, s)
            for s in lanes:
                if s is not root:
                    root.wait_stream(s)
        self.graph, self.plan = g, plan
        return g

    def replay(self) -> None:
        self.graph.replay()

    def _time(self, fn, reps: int = 3) -> float:
        torch = self.torch
        fn()
        torch.cuda.synchronize(self.dev)
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) * 1e-3)
        return best

    def autotune(self, table: Optional[TuneTable] = None, candidates=(1, 2, 3, 4, 8)) -> Plan:
        """Pick and capture the fastest plan (see module docstring)."""
        torch = self.torch
        name = torch.cuda.get_device_name(self.dev)
        key = mix_key(self.counts, name)
        if table is not None:
            known = table.get(key)
            if (known is not None and sorted(x for l in known.streams for x in l) == sorted(self.counts)
                    and sorted(known.configs or {}) == sorted(self.counts)):
                try:
                    for n, cfg in known.configs.items():
                        self.use_config(n, cfg)
                except RuntimeError:
                    # a stored configuration this build cannot create (an older
                    # table, another regime limit): tune again and overwrite it
                    known = None
                if known is not None:
                    self.capture(known)
                    return known
        from .solver import Solver
        cur = torch.cuda.current_stream(self.dev)
        cost = {}
        for n in self.counts:                      # per size: fastest execution config on its own data
            best_cfg, best_t = None, float("inf")
            for cfg in size_configs(n):
                try:
                    cand = Solver(n, device_id=self.dev.index or 0, regime=cfg["regime"],
                                  slots_per_sm=cfg["slots_per_sm"])
                except RuntimeError:               # this config cannot hold n
                    continue
                try:
                    t = self._time(lambda: cand.launch(self.H[n], self.S[n], self.W[n], self.U[n],
                                                       self.info[n], cur), reps=2)
                finally:
                    cand.close()
                if t < best_t:
                    best_cfg, best_t = cfg, t
            self.use_config(n, best_cfg)
            cost[n] = best_t
        best, best_t = None, float("inf")
        seen = set()
        for k in candidates:
            plan = lpt_plan(cost, k)
            sig = json.dumps(plan.streams)
            if sig in seen:
                continue
            seen.add(sig)
            self.capture(plan)
            t = self._time(self.replay, reps=3)
            if t < best_t:
                best, best_t = plan, t
        best.configs = dict(self.configs)
        self.capture(best)
        if table is not None:
            table.put(key, best)
        return best


    # ---------------------------------------------------------------- persistent form
    def persistent(self, configs: Optional[Dict[int, dict]] = None) -> None:
        """(Re)create the one-launch solver with per-size configurations
        {n: {"regime": ..., "per_item": ...}} (missing sizes: library defaults)
        and drop any captured graph of the previous one."""
        from .solver import UnevenSolver
        configs = configs or {}
        if len(self.counts) > 8:
            raise ValueError("the persistent form takes at most 8 sizes")
        old = self.uneven
        self.pgraph = None
        self.uneven = UnevenSolver(list(self.counts), device_id=self.dev.index or 0,
                                   regimes={n: c.get("regime") for n, c in configs.items()},
                                   per_item={n: c.get("per_item") for n, c in configs.items()})
        if old is not None:
            self.torch.cuda.synchronize(self.dev)
            old.close()
        self.pconfigs = {n: {"regime": r, "per_item": p} for n, r, p in self.uneven.shape}

    def launch_persistent(self, stream=None) -> None:
        """One launch of the persistent kernel over the whole mix."""
        if self.uneven is None:
            self.persistent()
        self.uneven.launch(self.H, self.S, self.W, self.U, self.info, stream)

    def capture_persistent(self):
        torch = self.torch
        if self.uneven is None:
            self.persistent()
        s = self._lane_streams(Plan([[0]]))[0]
        s.wait_stream(torch.cuda.current_stream(self.dev))
        self.launch_persistent(s)                      # warm-up on the capture stream
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.launch_persistent(s)
        self.pgraph = g
        return g

    def replay_persistent(self) -> None:
        if self.pgraph is None:
            self.capture_persistent()
        self.pgraph.replay()

    def autotune_persistent(self, table: Optional[TuneTable] = None, per_item_choices=(1, 4, 16)) -> Dict[int, dict]:
        """Choose each size's regime and problems per item for the one-launch
        form (see module docstring); remembered per size mix in `table`."""
        torch = self.torch
        key = "persistent|" + mix_key(self.counts, torch.cuda.get_device_name(self.dev))
        if table is not None:
            known = table.get(key)
            if known is not None and sorted(known.persistent or {}) == sorted(self.counts):
                try:
                    self.persistent(known.persistent)
                    self.capture_persistent()
                    return dict(self.pconfigs)
                except RuntimeError:
                    pass                                  # a choice this build cannot make: tune again
        self.persistent()
        best = dict(self.pconfigs)
        best_t = self._time(self.launch_persistent, reps=2)
        for n in sorted(self.counts, key=lambda x: -x):
            cands = []
            regimes = ["smem-cta", "l2-slot"] if n <= 64 else ["l2-slot"]
            for r in regimes:
                for p in (per_item_choices if r == "smem-cta" else (1,)):
                    cands.append({"regime": r, "per_item": p})
            for c in cands:
                if c == best[n]:
                    continue
                trial = dict(best)
                trial[n] = c
                try:
                    self.persistent(trial)
                except RuntimeError:
                    continue
                t = self._time(self.launch_persistent, reps=2)
                if t < best_t:
                    best, best_t = dict(self.pconfigs), t
        self.persistent(best)
        self.capture_persistent()
        if table is not None:
            table.put(key, Plan([sorted(self.counts)], persistent=dict(self.pconfigs)))
        return dict(self.pconfigs)
