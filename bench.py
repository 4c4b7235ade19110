#!/usr/bin/env python
"""Benchmark: batched generalized eigensolves H u = lambda S u (complex128).

One step = one sunny_geneig_launch over the whole batch (default N=54,
batch 65,536, the baseline generator with cond(S) <= 100), inputs resident
in HBM (6.1 GB of H and S, far larger than the 126 MB L2, so no flush is
needed between steps). Prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--n 54] [--batch 65536]
  python bench.py --impl reference ...   # LAPACK zhegv on the host cores

Multi-GPU (torchrun, one process per GPU): every rank solves its own
batch (weak scaling, replicas; the path has no exchange step), the timed
region is bracketed by barriers and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "N=54 gen-eig solves/s at ≤1e-12 residual, FP64 vs mixed; serving p50/p99 ms"


def flops_per_solve(n: int) -> float:
    # potrf 4/3 n^3 + hegst 4 n^3 + hetrd 16/3 n^3 + unmtr 8 n^3 + back-trsm 4 n^3 (real flops)
    return 68.0 / 3.0 * n ** 3


def hbm_bytes_per_solve(n: int, sigma: bool = False) -> int:
    # read H, S; write U (16 B each), W (8 B), info (4 B); the metric solve
    # never reads H
    return (32 if sigma else 48) * n * n + 8 * n + 4


def eig_err_vs_zhegv(H, S, W, n_sample: int = 512, seed: int = 20261206) -> dict:
    """Eigenvalues of a fixed random sample of the bench's matrices against
    LAPACK zhegv (scipy's OpenBLAS, itype=1, jobz='N', uplo='L') on the host:
    max |W - W_zhegv| / ||H||_2 over the sample. H, S, W are the device
    buffers in column-major layout (H[b] holds matrix b transposed)."""
    import numpy as np
    from scipy.linalg import lapack
    batch = W.shape[0]
    idx = np.sort(np.random.default_rng(seed).choice(batch, size=min(n_sample, batch), replace=False))
    import torch
    it = torch.from_numpy(idx).to(W.device)
    Hs = H.index_select(0, it).transpose(-1, -2).cpu().numpy()
    Ss = S.index_select(0, it).transpose(-1, -2).cpu().numpy()
    Ws = W.index_select(0, it).cpu().numpy()
    worst = 0.0
    for b in range(len(idx)):
        w, _, inf = lapack.zhegv(Hs[b], Ss[b], itype=1, jobz="N", uplo="L")
        if inf != 0:
            return {"max_eig_err_vs_zhegv": None, "zhegv_info_nonzero": int(inf)}
        worst = max(worst, float(np.abs(Ws[b] - w).max() / np.linalg.norm(Hs[b], 2)))
    return {"max_eig_err_vs_zhegv": worst, "eig_check_sample": len(idx)}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--n", type=int, default=54)
    p.add_argument("--batch", type=int, default=65536)
    p.add_argument("--kappa", type=float, default=100.0)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--e2e-chunk", type=int, default=8192)
    p.add_argument("--kernel", choices=["unified", "mixed"], default="unified",
                   help="mixed: FP32 Householder reduction + FP64 Ogita-Aishima refinement (kernel mode 2)")
    p.add_argument("--sigma", action="store_true",
                   help="spin-wave metric pencils: H = diag(I, -I) implied (sunny_geneig_launch_sigma), "
                        "S = the BdG matrix")
    p.add_argument("--serving", action="store_true", help="run the serving-loop workload instead")
    p.add_argument("--uneven", action="store_true", help="run the uneven-size batch workload instead")
    p.add_argument("--uneven-total", type=int, default=200000, help="uneven: number of problems")
    p.add_argument("--rate", type=float, default=50.0, help="serving: Poisson arrival rate (req/s)")
    p.add_argument("--duration", type=float, default=10.0, help="serving: arrival window (s)")
    p.add_argument("--sizes", type=str, default="18,54,108,216,384", help="serving: matrix sizes")
    p.add_argument("--qmax", type=int, default=4096, help="serving: largest q-points per request")
    p.add_argument("--budget-gb", type=float, default=150.0, help="serving: device-memory budget")
    p.add_argument("--slots", type=int, default=8, help="serving: requests in flight (streams)")
    p.add_argument("--fourier", action="store_true",
                   help="run the fused-assembly workload instead: S(q) built on the device from the Fourier "
                        "terms of a seeded N/2-site spin-wave model, then the metric solve, in one launch")
    p.add_argument("--bonds", type=int, default=120, help="fourier: exchange bonds of the model")
    p.add_argument("--profile", action="store_true",
                   help="bracket the timed launches with cudaProfilerStart/Stop, so that a profiler "
                        "started with --profile-from-start off (ncu, nsys) captures only them")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.cpu_baseline import ZhegvPool
    # enough problems per worker that a step is ~0.25 s of LAPACK work at N=54,
    # so that the pool's per-step dispatch is a small part of the time
    per_worker = max(16, int(256 * (54.0 / args.n) ** 3))
    pool = ZhegvPool(args.n, per_worker=per_worker, kappa=args.kappa)
    solved_per_step = per_worker * pool.workers
    try:
        for _ in range(max(args.warmup, 1)):
            pool.step()
        total, wall = 0, 0.0
        for _ in range(args.steps):
            s, t = pool.step()
            total += s
            wall += t
    finally:
        pool.close()
    value = total / wall
    cpu = {"value": value, "unit": "solves/s", "cores": pool.workers, "kind": "port",
           "sample": (f"each step: {pool.workers} single-threaded LAPACK zhegv workers (scipy OpenBLAS) "
                      f"solve their own {per_worker} seeded N={args.n} problems; {total} solves in {wall:.2f} s")}
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(args, world), reference_solves_per_step=solved_per_step,
                       reference_sample=(f"each step solves {solved_per_step} problems of this workload's "
                                         f"distribution ({pool.workers} workers x {per_worker}), not the "
                                         f"whole batch")),
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("the reference's GPU paths need NVIDIA MathDx/cuSolverDx, absent offline; its own CPU "
                 "ground truth (LAPACK zhegv) is timed instead"),
    }
    print(json.dumps(out), flush=True)


def workload_config(args, world):
    return {
        "workload": (f"N={args.n} complex128 spin-wave metric pencils (diag(I, -I), S), batch {args.batch} "
                     f"per GPU, S = BdG-structured PD matrix (lambda_min = 0.1 ||S||); H implied, not read; "
                     f"one launch per step" if getattr(args, "sigma", False) else
                     f"N={args.n} complex128 Hermitian-definite pairs, batch {args.batch} per GPU, "
                     f"BdG-structured H (lambda_min = 0.1 ||H||), S = Q diag(d) Q^H with cond(S) <= "
                     f"{args.kappa:g}; one launch per step"),
        "n": args.n, "batch_per_gpu": args.batch, "global_batch": args.batch * world,
        "cond_S_max": args.kappa, "parallelism": f"replicas x{world}",
        "kernel": getattr(args, "kernel", "unified"),
        "l2": "inputs 2 x batch x N^2 x 16 B >> 126 MB L2 (no flush needed)"
        if 2 * args.batch * args.n * args.n * 16 > 126e6 else "inputs fit L2: L2 flushed between steps",
    }


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd[1:1] = ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------- our arm
def measure_fp64_peak(torch, dev) -> float:
    """cuBLAS DGEMM TFLOP/s (torch.matmul float64, 8192^3), best of 4."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def run_ours(args):
    rank, world, local = dist_env()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle.cpu_baseline import time_zhegv   # CPU baseline leg (spawned before any CUDA use)
        cpu = time_zhegv(args.n, per_worker=32, seconds=8.0, kappa=args.kappa)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from sunny_gen_eigensolver_b200 import Solver, replicas
    from sunny_gen_eigensolver_b200.generators import baseline_problems_torch

    n, batch = args.n, args.batch
    H, S = baseline_problems_torch(n, batch, seed=replicas.rank_seed(20261203 + 1, rank), kappa=args.kappa,
                                   device=dev)
    if args.sigma:
        # Sunny's pattern: the PD BdG matrix is the metric-side S, H = diag(I, -I)
        sig = torch.cat([torch.ones(n // 2), -torch.ones(n - n // 2)]).to(torch.complex128)
        S, H = H, torch.diag(sig).to(dev).expand(batch, n, n).contiguous()
    # column-major buffers (Julia layout), transposed in place chunk by chunk
    # so that a 1M-problem batch never holds a second full copy
    for X in (H, S):
        for c0 in range(0, batch, 65536):
            blk = X[c0:c0 + 65536]
            blk.copy_(blk.transpose(-1, -2).contiguous())
    W = torch.empty((batch, n), dtype=torch.float64, device=dev)
    U = torch.empty((batch, n, n), dtype=torch.complex128, device=dev)
    info = torch.empty((batch,), dtype=torch.int32, device=dev)
    solver = Solver(n, device_id=local, kernel=args.kernel)
    stream = torch.cuda.current_stream(dev)

    peak = measure_fp64_peak(torch, dev)

    def barrier():
        replicas.barrier(dev)

    def do_launch(Hx, Sx, Wx, Ux, ix, st):
        if args.sigma:
            solver.launch_sigma(Sx, Wx, Ux, ix, st)
        else:
            solver.launch(Hx, Sx, Wx, Ux, ix, st)

    for _ in range(args.warmup):
        do_launch(H, S, W, U, info, stream)
    barrier()
    props = torch.cuda.get_device_properties(dev)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None)
    with ClockSampler(uuid) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        if args.profile:
            torch.cuda.profiler.start()
        t0.record(stream)
        for _ in range(args.steps):
            do_launch(H, S, W, U, info, stream)
        t1.record(stream)
        barrier()
        if args.profile:
            torch.cuda.profiler.stop()
    elapsed = t0.elapsed_time(t1) * 1e-3
    elapsed_max = replicas.max_over_ranks(elapsed, dev)
    clocks = clk.summary()

    # accuracy of the last step's results (all matrices, on the device)
    bad = int((info != 0).sum().item())
    res_max, orth_max = 0.0, 0.0
    eye = torch.eye(n, dtype=torch.complex128, device=dev)
    for c0 in range(0, batch, 65536):        # chunked: the checks' temporaries stay a few GB
        sl = slice(c0, min(batch, c0 + 65536))
        Hn, Sn, Un = H[sl].transpose(-1, -2), S[sl].transpose(-1, -2), U[sl].transpose(-1, -2)
        R = Hn @ Un - (Sn @ Un) * W[sl, None, :].to(torch.complex128)
        hnorm_lb = torch.linalg.matrix_norm(Hn) / n ** 0.5        # ||H||_F / sqrt(n) <= ||H||_2
        unorm_lb = torch.linalg.matrix_norm(Un) / n ** 0.5        # ||U||_F / sqrt(n) <= ||U||_2
        res_max = max(res_max, float((torch.linalg.matrix_norm(R) / (hnorm_lb * unorm_lb)).max().item()))
        del R
        G = Un.conj().transpose(-1, -2) @ Sn @ Un - eye
        orth_max = max(orth_max, float(G.abs().amax().item()))
        del G
    acc = {"max_residual_upper_bound": res_max, "max_s_orth": orth_max,
           "failed_matrices": bad, "sorted": bool((W[:, 1:] >= W[:, :-1]).all().item())}
    if rank == 0:
        acc.update(eig_err_vs_zhegv(H, S, W))
    if args.kernel == "mixed":
        # eigenvalues against the plain FP64 kernel on the same inputs (that
        # kernel is held to LAPACK zhegv by the parity tests)
        Wp = torch.empty_like(W)
        Up = torch.empty_like(U)
        ip = torch.empty_like(info)
        with Solver(n, device_id=local) as sp:
            if args.sigma:
                sp.launch_sigma(S, Wp, Up, ip, stream)
            else:
                sp.launch(H, S, Wp, Up, ip, stream)
            torch.cuda.synchronize(dev)
        scale = Wp.abs().amax(dim=1).clamp_min(1e-300)
        acc["max_eig_diff_vs_plain_rel"] = float(((W - Wp).abs().amax(dim=1) / scale).max().item())
        del Wp, Up, ip

    solves = batch * world * args.steps
    value = solves / elapsed_max
    per_launch = elapsed / args.steps
    achieved = flops_per_solve(n) * batch / per_launch / 1e12
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 via torch.matmul (best of 4)",
                "traffic": None,
                "algorithmic_bytes_per_launch": hbm_bytes_per_solve(n, args.sigma) * batch,
                "achieved_hbm_gbs": hbm_bytes_per_solve(n, args.sigma) * batch / per_launch / 1e9}
    tfile = REPO / "profiles" / f"dram_traffic_n{n}.json"
    if tfile.exists() and not args.sigma:
        try:
            t = json.loads(tfile.read_text())
            roofline["traffic"] = t["dram_bytes_per_solve"] * batch
            roofline["traffic_source"] = t.get("source", str(tfile.name))
        except Exception:
            pass

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, torch, do_launch, H, S, W, U, info, dev, world, dist)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.kernel == "mixed" else "f64",
            "data": "synthetic (seeded BdG H / Haar-unitary S generator, generated on the device)",
            "config": workload_config(args, world),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": args.steps, "accuracy": acc,
            "solver": {"regime": solver.regime, "block_dim_x": solver.block_dim_x,
                       "shared_mem_bytes": solver.shared_mem_bytes, "path": solver.path_name},
        }
        print(json.dumps(out), flush=True)
    solver.close()
    if world > 1:
        dist.destroy_process_group()


def run_e2e(args, torch, do_launch, H, S, W, U, info, dev, world, dist):
    """Same metric through the C ABI with HOST buffers: every step copies H and
    S (S alone for the metric solve) in from pinned host memory and W, U, info
    back out, pipelined in chunks over three streams (H2D, launch and D2H of
    different chunks overlap)."""
    batch, n = args.batch, args.n
    Hh = H.cpu().pin_memory() if not args.sigma else None
    Sh = S.cpu().pin_memory()
    Wh = torch.empty(W.shape, dtype=W.dtype).pin_memory()
    Uh = torch.empty(U.shape, dtype=U.dtype).pin_memory()
    ih = torch.empty(info.shape, dtype=info.dtype).pin_memory()
    streams = [torch.cuda.Stream(dev) for _ in range(3)]
    chunk = args.e2e_chunk

    def step():
        for k, off in enumerate(range(0, batch, chunk)):
            sl = slice(off, min(batch, off + chunk))
            s = streams[k % len(streams)]
            with torch.cuda.stream(s):
                if Hh is not None:
                    H[sl].copy_(Hh[sl], non_blocking=True)
                S[sl].copy_(Sh[sl], non_blocking=True)
                do_launch(H[sl], S[sl], W[sl], U[sl], info[sl], s)
                Wh[sl].copy_(W[sl], non_blocking=True)
                Uh[sl].copy_(U[sl], non_blocking=True)
                ih[sl].copy_(info[sl], non_blocking=True)

    steps = max(3, args.steps // 2)
    for _ in range(2):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(dev)
    ev0.record(cur)
    for s in streams:
        s.wait_stream(cur)
    for _ in range(steps):
        step()
    for s in streams:
        cur.wait_stream(s)
    ev1.record(cur)
    torch.cuda.synchronize(dev)
    el = max(ev0.elapsed_time(ev1) * 1e-3, 1e-9)
    el_t = torch.tensor([el], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(el_t, op=dist.ReduceOp.MAX)
    el = float(el_t.item())
    bi = (1 if args.sigma else 2) * batch * n * n * 16
    bo = batch * (n * n * 16 + n * 8 + 4)
    return {"value": batch * world * steps / el, "unit": "solves/s", "h2d_bytes_per_step": bi,
            "d2h_bytes_per_step": bo, "steps": steps, "chunk": chunk, "streams": len(streams),
            "host_wall_s": time.perf_counter() - t0}


def run_fourier(args):
    """Fused dynamical-matrix assembly: per q-point, S(q) = sum_t coef_t
    exp(2 pi i q . d_t) is built in shared memory from the terms of a seeded
    spin-wave model (m = N/2 sites, --bonds exchange bonds, a field that gaps
    every mode) and solved as the metric pencil H = diag(I, -I) in the same
    launch (sunny_geneig_launch_fourier_sigma); S never exists in memory.
    Against it: the unfused two-step path (the assembly as torch index_add
    writing S to HBM, then sunny_geneig_launch_sigma reading it back)."""
    import numpy as np
    import torch
    from sunny_gen_eigensolver_b200 import Solver, lswt
    n, batch = args.n, args.batch
    m = n // 2
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    model = lswt.random_model(m, args.bonds, seed=20261208)
    rows, cols, coef, disp = lswt.fourier_terms(model)
    start, c, d = lswt.pack_terms(n, rows, cols, coef, disp)
    solver = Solver(n)
    terms = solver.device_terms(start, c, d)
    gen = torch.Generator(device=dev)
    gen.manual_seed(20261209)
    q = (torch.rand((batch, 3), generator=gen, dtype=torch.float64, device=dev) - 0.5).contiguous()
    W = torch.empty((batch, n), dtype=torch.float64, device=dev)
    U = torch.empty((batch, n, n), dtype=torch.complex128, device=dev)
    info = torch.empty((batch,), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    peak = measure_fp64_peak(torch, dev)

    def timed(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / k

    props = torch.cuda.get_device_properties(dev)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None)
    with ClockSampler(uuid) as clk:
        t_fused = timed(lambda: solver.launch_fourier_sigma(terms, q, W, U, info, stream), args.steps)
    clocks = clk.summary()
    bad = int((info != 0).sum().item())

    # unfused: the same assembly in torch (S to HBM, column-major), then the metric solve
    lower = np.asarray(rows) >= np.asarray(cols)
    ent = torch.from_numpy((np.asarray(rows) + n * np.asarray(cols))[lower]).to(dev)
    cf = torch.from_numpy(np.asarray(coef)[lower]).to(dev)
    dp = torch.from_numpy(np.asarray(disp)[lower]).to(dev)
    S = torch.zeros((batch, n, n), dtype=torch.complex128, device=dev)
    W2, U2, info2 = torch.empty_like(W), torch.empty_like(U), torch.empty_like(info)
    chunk = 8192

    def assemble():
        Sv = S.view(batch, n * n)
        for c0 in range(0, batch, chunk):
            x = 2 * np.pi * (q[c0:c0 + chunk] @ dp.T)
            ph = torch.complex(torch.cos(x), torch.sin(x)) * cf
            Sv[c0:c0 + chunk].zero_().index_add_(1, ent, ph)

    def unfused():
        assemble()
        solver.launch_sigma(S, W2, U2, info2, stream)

    t_unfused = timed(unfused, max(1, args.steps // 2))
    # S is column-major with the lower triangle filled: mirror it for the host check
    Sn = S.transpose(-1, -2)
    Sfull = torch.tril(Sn) + torch.tril(Sn, -1).conj().transpose(-1, -2)
    sig = torch.diag(torch.cat([torch.ones(m), -torch.ones(m)]).to(torch.complex128)).to(dev)
    Hc = sig.expand(batch, n, n)
    acc = {"failed_matrices": bad, "sorted": bool((W[:, 1:] >= W[:, :-1]).all().item()),
           "max_eig_diff_fused_vs_unfused": float((W - W2).abs().max().item())}
    acc.update(eig_err_vs_zhegv(Hc.transpose(-1, -2), Sfull.transpose(-1, -2), W))
    res_max, orth_max = 0.0, 0.0
    eye = torch.eye(n, dtype=torch.complex128, device=dev)
    for c0 in range(0, batch, chunk):
        sl = slice(c0, min(batch, c0 + chunk))
        Un = U[sl].transpose(-1, -2)
        Sl = Sfull[sl]
        R = sig @ Un - (Sl @ Un) * W[sl, None, :].to(torch.complex128)
        unorm_lb = torch.linalg.matrix_norm(Un) / n ** 0.5
        res_max = max(res_max, float((torch.linalg.matrix_norm(R) / unorm_lb).max().item()))
        orth_max = max(orth_max, float((Un.conj().transpose(-1, -2) @ Sl @ Un - eye).abs().amax().item()))
    acc.update({"max_residual_upper_bound": res_max, "max_s_orth": orth_max})
    del S, Sfull, Sn

    # e2e through the C ABI: q in from pinned host memory, W, U, info out
    qh = q.cpu().pin_memory()
    Wh = torch.empty(W.shape, dtype=W.dtype).pin_memory()
    Uh = torch.empty(U.shape, dtype=U.dtype).pin_memory()
    ih = torch.empty(info.shape, dtype=info.dtype).pin_memory()
    streams = [torch.cuda.Stream(dev) for _ in range(3)]

    def step():
        for k, off in enumerate(range(0, batch, chunk)):
            sl = slice(off, min(batch, off + chunk))
            st = streams[k % len(streams)]
            with torch.cuda.stream(st):
                q[sl].copy_(qh[sl], non_blocking=True)
                solver.launch_fourier_sigma(terms, q[sl], W[sl], U[sl], info[sl], st)
                Wh[sl].copy_(W[sl], non_blocking=True)
                Uh[sl].copy_(U[sl], non_blocking=True)
                ih[sl].copy_(info[sl], non_blocking=True)

    for _ in range(2):
        step()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(dev)
    e2e_steps = max(3, args.steps // 2)
    ev0.record(cur)
    for st in streams:
        st.wait_stream(cur)
    for _ in range(e2e_steps):
        step()
    for st in streams:
        cur.wait_stream(st)
    ev1.record(cur)
    torch.cuda.synchronize(dev)
    el = ev0.elapsed_time(ev1) * 1e-3
    e2e = {"value": batch * e2e_steps / el, "unit": "solves/s", "h2d_bytes_per_step": batch * 24,
           "d2h_bytes_per_step": batch * (n * n * 16 + n * 8 + 4), "steps": e2e_steps, "chunk": chunk,
           "streams": len(streams)}

    achieved = flops_per_solve(n) * batch / t_fused / 1e12
    out = {"metric": METRIC, "mode": "fourier", "value": batch / t_fused, "unit": "solves/s",
           "ms_per_step": 1e3 * t_fused, "steps": args.steps, "warmup": args.warmup, "n_gpus": 1,
           "higher_is_better": True, "dtype": "f64",
           "data": "synthetic (seeded spin-wave model, uniform random q)",
           "config": {"workload": f"N={n} spin-wave metric solve, S(q) assembled on the device "
                                  f"({m} sites, {args.bonds} bonds, {int(c.shape[0])} lower-triangle terms)",
                      "n": n, "batch": batch, "terms": int(c.shape[0])},
           "unfused_solves_per_s": batch / t_unfused, "fused_vs_unfused": t_unfused / t_fused,
           "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak, "traffic": None,
                        "algorithmic_bytes_per_launch": batch * (24 + n * n * 16 + n * 8 + 4)},
           "e2e": e2e, "clocks": clocks, "gpu_launches": args.steps, "accuracy": acc,
           "solver": {"regime": solver.regime, "block_dim_x": solver.block_dim_x}}
    print(json.dumps(out), flush=True)
    solver.close()


def run_serving(args):
    """Serving workload: Poisson request arrivals, each request q log-uniform
    q-points of one N, admitted by a device-memory budget, overlapped on a
    stream pool; prints one JSON line with p50/p99 latency and solves/s."""
    import torch
    from sunny_gen_eigensolver_b200.serving import DeviceExecutor, ServingEngine, poisson_requests
    sizes = [int(x) for x in args.sizes.split(",")]
    reqs = poisson_requests(args.rate, args.duration, sizes, q_range=(64, args.qmax), seed=20261207)
    ex = DeviceExecutor(slots=args.slots, pool_size=256, kernel=args.kernel)
    ex.prepare(sizes)
    # the budget covers the admitted requests' state; keep 8 GB of the free
    # memory for the input pools' gathers and the allocator's slack
    free, _ = torch.cuda.mem_get_info()
    budget = int(min(args.budget_gb * 1e9, free - 8e9))
    failed = [0]

    def consume(r, res):          # the client reads its answer; nothing is kept
        failed[0] += int((res[2] != 0).sum().item())

    warm = poisson_requests(1000.0, 0.01, sizes, q_range=(8, 16), seed=1)
    ServingEngine(ex, budget_bytes=budget, consume=consume).run(warm)     # warm-up
    torch.cuda.synchronize()
    failed[0] = 0
    st = ServingEngine(ex, budget_bytes=budget, consume=consume).run(reqs)
    torch.cuda.synchronize()
    bad = failed[0]
    # the arrival process is sustainable when the queue stays short: no request
    # waited behind more than a few others
    sustained = st.max_waiting <= 2 * args.slots
    out = {"metric": METRIC, "mode": "serving", "value": st.solves_per_s, "unit": "solves/s",
           "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms, "n_gpus": 1,
           "kernel": args.kernel,
           "latency_bound": (f"p99 <= {st.p99_ms:.1f} ms at {args.rate:g} req/s ({args.kernel} form, sizes "
                             f"{args.sizes}, q 64..{args.qmax})" if sustained else
                             f"not sustained: the queue grew to {st.max_waiting} requests at {args.rate:g} req/s"),
           "higher_is_better": True, "dtype": "f32+f64" if args.kernel == "mixed" else "f64",
           "data": "synthetic (seeded per-N device pools)",
           "config": {"workload": "serving loop", "rate_hz": args.rate, "duration_s": args.duration,
                      "sizes": sizes, "q_range": [64, args.qmax], "budget_gb": budget / 1e9,
                      "slots": args.slots, "requests": len(reqs)},
           "stats": st.as_dict(), "failed_matrices": bad,
           "solver_regimes": {n: ex.solvers[n].regime for n in sizes}}
    print(json.dumps(out), flush=True)


def run_uneven(args):
    """Uneven-size batch: problems with N drawn from {12,24,54,72,108,162,216}
    (30/20/25/10/8/5/2 %), packed per size, all sizes in one CUDA graph launch
    (autotuned stream plan) vs one plain launch per size on one stream."""
    import numpy as np
    import torch
    from sunny_gen_eigensolver_b200.batching import TuneTable, UnevenBatch
    from sunny_gen_eigensolver_b200.generators import baseline_problems_torch
    sizes_set = [12, 24, 54, 72, 108, 162, 216]
    weights = [0.30, 0.20, 0.25, 0.10, 0.08, 0.05, 0.02]
    rng = np.random.default_rng(20261205)
    sizes = rng.choice(sizes_set, size=args.uneven_total, p=weights)
    ub = UnevenBatch(sizes)
    for n, c in ub.counts.items():
        H, S = baseline_problems_torch(n, c, seed=3000 + n, kappa=args.kappa)
        ub.set_inputs(n, H.transpose(-1, -2), S.transpose(-1, -2))
        del H, S
    torch.cuda.synchronize()
    table = TuneTable(Path(tempfile.gettempdir()) / "sunny_geneig_bench_plans.json")
    plan = ub.autotune(table)

    def timed(fn, k):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / k

    steps = max(1, args.steps // 4)
    t_graph = timed(ub.replay, steps)
    t_seq = timed(ub.run_sequential, steps)
    # the persistent form: one kernel launch for the whole mix, per-size regime
    # and problems per work item autotuned, replayed from a captured graph
    pconf = ub.autotune_persistent(table)
    t_pers = timed(ub.replay_persistent, steps)
    # one plain launch per size with the library's default configuration per N
    from sunny_gen_eigensolver_b200 import Solver
    defaults = {n: Solver(n) for n in ub.counts}
    cur = torch.cuda.current_stream()

    def run_default():
        for n, s in defaults.items():
            s.launch(ub.H[n], ub.S[n], ub.W[n], ub.U[n], ub.info[n], cur)

    t_def = timed(run_default, steps)
    for s in defaults.values():
        s.close()
    ub.replay_persistent()             # leave the persistent form's results in the buffers for the checks
    torch.cuda.synchronize()
    bad = sum(int((ub.info[n] != 0).sum().item()) for n in ub.counts)
    flops = sum(flops_per_solve(n) * c for n, c in ub.counts.items())
    out = {"metric": METRIC, "mode": "uneven", "value": ub.total / t_pers, "unit": "solves/s",
           "ms_per_step": 1e3 * t_pers, "steps": steps, "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
           "data": "synthetic (seeded BdG H / Haar-unitary S per size)",
           "config": {"workload": "uneven-size persistent batch (one kernel launch, graph replay)",
                      "total": ub.total, "counts": {str(n): c for n, c in ub.counts.items()}},
           "persistent_solves_per_s": ub.total / t_pers,
           "persistent_configs": {str(n): c for n, c in pconf.items()},
           "persistent_vs_default_per_size_launches": t_def / t_pers,
           "graph_solves_per_s": ub.total / t_graph, "sequential_solves_per_s": ub.total / t_seq,
           "graph_speedup": t_seq / t_graph, "plan_streams": plan.streams,
           "sequential_default_config_solves_per_s": ub.total / t_def,
           "size_configs": {str(n): c for n, c in (plan.configs or {}).items()},
           "achieved_fp64_tflops": flops / t_pers / 1e12, "failed_matrices": bad,
           "regimes": {str(n): ub.solvers[n].regime for n in ub.counts}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.serving:
        run_serving(args)
    elif args.uneven:
        run_uneven(args)
    elif args.fourier:
        run_fourier(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
