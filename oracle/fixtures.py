"""GEIG v1 fixture format and the reference's seeded fixture generator.

Format (the reference's tests/common/lapack_reference.cpp:256-283, read by
dump_pair.cpp:41-71): six little-endian int32 {0x47454947 'GEIG', 1, N, B,
seed, 0}, then H[B], S[B] (column-major complex128 N x N each), W[B*N]
(float64), U[B] (column-major complex128). Arrays returned here are in
natural layout (batch, n, n) with M[b, i, j] = entry (i, j).

`generate(n, batch, seed, mode)` calls the C++ restatement of the
reference generator (fixture_gen.cpp, built into oracle/_build/ by
`build()`), which reproduces the fixtures' H and S bit-for-bit.
"""
from __future__ import annotations

import ctypes
import struct
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
BUILD_DIR = ORACLE_DIR / "_build"
GEN_LIB = BUILD_DIR / "libgeig_fixture.so"
MAGIC, VERSION = 0x47454947, 1


def build(force: bool = False) -> Path:
    src = ORACLE_DIR / "fixture_gen.cpp"
    if force or not GEN_LIB.exists() or GEN_LIB.stat().st_mtime < src.stat().st_mtime:
        BUILD_DIR.mkdir(exist_ok=True)
        tmp = GEN_LIB.with_suffix(".so.tmp")
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", str(tmp), str(src)], check=True)
        tmp.replace(GEN_LIB)
    return GEN_LIB


_gen = None


def _lib():
    global _gen
    if _gen is None:
        build()
        _gen = ctypes.CDLL(str(GEN_LIB))
        _gen.geig_fixture_generate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_void_p]
        _gen.geig_fixture_generate.restype = ctypes.c_int
    return _gen


def generate(n: int, batch: int, seed: int, mode: str = "random"):
    """(H, S) exactly as the reference's lapack_reference --s-mode {random,near-identity}."""
    m = {"random": 0, "nearid": 1, "near-identity": 1}[mode]
    Hc = np.zeros(n * n * batch, dtype=np.complex128)
    Sc = np.zeros(n * n * batch, dtype=np.complex128)
    rc = _lib().geig_fixture_generate(n, batch, seed, m, Hc.ctypes.data, Sc.ctypes.data)
    if rc:
        raise ValueError("bad fixture generator arguments")
    H = Hc.reshape(batch, n, n).transpose(0, 2, 1).copy()
    S = Sc.reshape(batch, n, n).transpose(0, 2, 1).copy()
    return H, S


def read_geig(path):
    with open(path, "rb") as f:
        magic, ver, n, b, seed, _ = struct.unpack("<6i", f.read(24))
        if magic != MAGIC or ver != VERSION:
            raise ValueError(f"{path}: not a GEIG v1 file")
        def cm(k):
            return np.frombuffer(f.read(16 * n * n * b), dtype=np.complex128).reshape(b, n, n).transpose(0, 2, 1).copy()
        H, S = cm(0), cm(1)
        W = np.frombuffer(f.read(8 * n * b), dtype=np.float64).reshape(b, n).copy()
        U = cm(3)
    return dict(n=n, batch=b, seed=seed, H=H, S=S, W=W, U=U)


def write_geig(path, H, S, W, U, seed: int) -> None:
    b, n, _ = H.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<6i", MAGIC, VERSION, n, b, seed, 0))
        for M in (H, S):
            f.write(np.ascontiguousarray(M.transpose(0, 2, 1)).astype(np.complex128).tobytes())
        f.write(np.ascontiguousarray(W, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(U.transpose(0, 2, 1)).astype(np.complex128).tobytes())
