"""Builds libsunny_geneig.so in-tree for sm_100a with nvcc.

The library is the product: the C ABI of include/sunny_geneig.h over the
hand-written kernels in csrc/. It is built in place (next to this file, in
lib/) so that it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
REPO_DIR = PKG_DIR.parent
CSRC = PKG_DIR / "csrc"
LIB_DIR = PKG_DIR / "lib"
LIB_PATH = LIB_DIR / "libsunny_geneig.so"
# profiling variant: same kernels with the clock64 phase timers compiled in
TIMERS_LIB_PATH = LIB_DIR / "libsunny_geneig_timers.so"
INCLUDE = REPO_DIR / "include"

SOURCES = ["geneig_cta.cu", "geneig_plain.cu", "geneig_tiled.cu", "geneig_uneven.cu", "selftest.cu", "tune.cu",
           "c_api.cpp"]
HEADERS = ["geneig_common.cuh", "geneig_dc.cuh", "geneig_kernels.h", "geneig_cta_body.cuh", "geneig_tiled_body.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(lib: Path = LIB_PATH) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [INCLUDE / "sunny_geneig.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False,
          phase_timers: bool = False) -> Path:
    """Compile the sources into lib/libsunny_geneig.so (skipped when up to date).

    `phase_timers` builds the profiling variant lib/libsunny_geneig_timers.so
    instead (-DSGEIG_PHASE_TIMERS: per-phase clock64 counters, read with
    sunny_geneig_phase_cycles; see phase_timers.py)."""
    lib = TIMERS_LIB_PATH if phase_timers else LIB_PATH
    if not force and not _stale(lib):
        return lib
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    objs, cmds = [], []
    extra = ["-DSGEIG_PHASE_TIMERS"] if phase_timers else []
    for src in SOURCES:
        obj = LIB_DIR / (Path(src).stem + (".timers.o" if phase_timers else ".o"))
        cmd = [_nvcc(), *NVCC_FLAGS, *extra, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / src), "-o", str(obj)]
        if ptxas_verbose and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args, r.stdout, r.stderr)
    tmp = lib.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *objs,
           "-Xcompiler", "-fvisibility=hidden"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    for o in objs:
        Path(o).unlink(missing_ok=True)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv,
                phase_timers="--phase-timers" in sys.argv))
