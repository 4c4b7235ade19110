"""Per-phase cycle split of the solver kernels (profiling aid).

Builds (if needed) and loads the profiling variant of the library,
lib/libsunny_geneig_timers.so, whose kernels (smem-cta and l2-slot) carry
clock64 marks after their CTA barriers (phase_mark in
csrc/geneig_common.cuh), runs a seeded batch through the size's default
kernel, and prints the CTA cycles per solve spent in each phase.

  python -m sunny_gen_eigensolver_b200.phase_timers [--n 54] [--batch 8192] [--reps 3]

Must run in a fresh process: it points the package's ctypes binding at the
profiling library before anything loads the product library.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

from . import build as _build

#: phase slot -> name (slots of geneig_cta.cu and geneig_dc.cuh)
PHASES = {
    0: "a1 load H, S", 1: "a2 Cholesky + L^-1", 2: "a3 T = H X^H", 3: "a4 C = X T",
    4: "a5a Householder tridiagonalisation", 5: "a5b D&C tail (finite check)",
    6: "a5c rank + back-transform V = Q Z", 7: "a6 U = X^H V", 8: "a7 store U (+ loop barrier)",
    10: "D&C scale + leaves", 11: "D&C deflation (phase A)", 12: "D&C secular roots (phase B)",
    13: "D&C Loewner z (phase C)", 14: "D&C rank-one vectors (phase D)", 15: "D&C merge GEMMs (phase E)",
    # l2-slot (tiled) kernel
    16: "tiled a1 load S", 17: "tiled a2 blocked Cholesky", 18: "tiled a3 X = L^-1",
    19: "tiled a4 T = H X^H, C = X T", 20: "tiled a5a Householder", 21: "tiled a5b D&C tail + rank",
    22: "tiled a5c WY back-transform (+ mixed refinement)", 23: "tiled a6 U = X^H V",
    24: "tiled a7 store U (+ loop barrier)",
}
#: event-counter slots (counts, not cycles)
COUNTERS = {27: "D&C secular iterations", 28: "D&C secular iterations, slowest root per level",
            29: "D&C secular roots solved"}


def main(argv=None) -> dict:
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=54)
    p.add_argument("--batch", type=int, default=8192)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--kappa", type=float, default=100.0)
    p.add_argument("--lib", type=str, default=None,
                   help="an already built profiling library to load instead of building lib/'s")
    args = p.parse_args(argv)

    lib = args.lib or _build.build(phase_timers=True)
    os.environ["SUNNY_GENEIG_LIBPATH"] = str(lib)
    import torch
    from . import _native
    from .generators import baseline_problems_torch
    from .solver import Solver

    L = _native.load()
    L.sunny_geneig_phase_cycles.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int, ctypes.c_int]
    L.sunny_geneig_phase_cycles.restype = ctypes.c_int
    H, S = baseline_problems_torch(args.n, args.batch, seed=20261203 + 1, kappa=args.kappa)
    H = H.transpose(-1, -2).contiguous()
    S = S.transpose(-1, -2).contiguous()
    W = torch.empty((args.batch, args.n), dtype=torch.float64, device=H.device)
    U = torch.empty_like(H)
    info = torch.empty((args.batch,), dtype=torch.int32, device=H.device)
    buf = (ctypes.c_ulonglong * 32)()
    with Solver(args.n) as s:
        s.launch(H, S, W, U, info)                     # warm-up
        L.sunny_geneig_phase_cycles(buf, 32, 1)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.reps):
            s.launch(H, S, W, U, info)
        ev1.record()
        torch.cuda.synchronize()
        if L.sunny_geneig_phase_cycles(buf, 32, 1) != 0:
            raise RuntimeError("reading the phase counters failed")
        regime = s.regime
    solves = args.batch * args.reps
    per = {PHASES.get(k, f"slot {k}"): buf[k] / solves for k in range(32) if buf[k] and k not in COUNTERS}
    counts = {name: buf[k] / solves for k, name in COUNTERS.items() if buf[k]}
    total = sum(per.values())
    out = {"n": args.n, "batch": args.batch, "reps": args.reps, "regime": regime,
           "failed": int((info != 0).sum().item()),
           "solves_per_s_timers_build": solves / (ev0.elapsed_time(ev1) * 1e-3),
           "cycles_per_solve_per_cta": {k: round(v) for k, v in per.items()}, "total_cycles": round(total),
           "counts_per_solve": {k: round(v, 2) for k, v in counts.items()}}
    for k, v in per.items():
        print(f"{k:42s} {v:10.0f}  {100 * v / total:5.1f} %", file=sys.stderr)
    for k, v in counts.items():
        print(f"{k:50s} {v:10.2f} per solve", file=sys.stderr)
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
