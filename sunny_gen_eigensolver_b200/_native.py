"""ctypes binding of libsunny_geneig.so (include/sunny_geneig.h).

The argument and return types below are the ones the reference's Julia
wrapper declares in its `ccall`s (julia/SunnyGeneigBench/src/SunnyGeneigBench.jl:
create_ex :48-51, launch :164-168, accessors :69-92): Cint arguments, device
pointers and the stream as unsigned machine words, an opaque handle.

There is no fallback: if the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
DEFAULT_LIB = _PKG / "lib" / "libsunny_geneig.so"

# enums (include/sunny_geneig.h)
STATUS_OK, STATUS_INVALID_ARG, STATUS_DEVICE_ERROR, STATUS_COMPILE_ERROR, STATUS_LAUNCH_ERROR = 0, -1, -2, -3, -4
CACHE_AUTO, CACHE_NODISK, CACHE_NOCACHE = 0, 1, 2
TUNING_SUGGESTED, TUNING_AUTOTUNE = 0, 1
KERNEL_UNIFIED, KERNEL_HYBRID, KERNEL_MIXED = 0, 1, 2

#: every symbol include/sunny_geneig.h declares
EXPORTS = (
    "sunny_geneig_create", "sunny_geneig_create_ex", "sunny_geneig_destroy", "sunny_geneig_launch",
    "sunny_geneig_matrix_size", "sunny_geneig_batches_per_block", "sunny_geneig_block_dim_x",
    "sunny_geneig_shared_mem_bytes", "sunny_geneig_last_error", "sunny_geneig_path_name",
    "sunny_geneig_kernel_mode", "sunny_geneig_launch_stage", "sunny_geneig_max_matrix_size",
    "sunny_geneig_regime_name", "sunny_geneig_selftest_reciprocal", "sunny_geneig_launch_noalloc",
    "sunny_geneig_launch_sigma", "sunny_geneig_create_config", "sunny_geneig_launch_sigma_intensity",
    "sunny_geneig_uneven_create", "sunny_geneig_uneven_launch", "sunny_geneig_uneven_destroy",
    "sunny_geneig_uneven_shape", "sunny_geneig_launch_fourier_sigma",
    "sunny_geneig_launch_fourier_sigma_intensity",
)

_lib = None


def lib_path() -> Path:
    env = os.environ.get("SUNNY_GENEIG_LIBPATH")
    return Path(env) if env else DEFAULT_LIB


def load() -> ctypes.CDLL:
    """Load (once) and type the shared library. Raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(
            f"libsunny_geneig.so not found at {path}; build it with "
            "`python -m sunny_gen_eigensolver_b200.build` (no CPU fallback exists)")
    L = ctypes.CDLL(str(path))
    c_int, c_uint, c_void_p, c_char_p, c_size = ctypes.c_int, ctypes.c_uint, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t
    L.sunny_geneig_create.argtypes = [c_int] * 5
    L.sunny_geneig_create.restype = c_void_p
    L.sunny_geneig_create_ex.argtypes = [c_int] * 6
    L.sunny_geneig_create_ex.restype = c_void_p
    L.sunny_geneig_create_config.argtypes = [c_int, c_int, c_int, ctypes.c_char_p, c_int]
    L.sunny_geneig_create_config.restype = c_void_p
    L.sunny_geneig_destroy.argtypes = [c_void_p]
    L.sunny_geneig_destroy.restype = None
    L.sunny_geneig_launch.argtypes = [c_void_p, c_size, c_size, c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch.restype = c_int
    L.sunny_geneig_launch_stage.argtypes = [c_void_p, c_int, c_size, c_size, c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_stage.restype = c_int
    L.sunny_geneig_launch_sigma.argtypes = [c_void_p, c_size, c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_sigma.restype = c_int
    L.sunny_geneig_launch_sigma_intensity.argtypes = [c_void_p, c_size, c_size, c_size, c_size, c_int,
                                                      ctypes.c_double, c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_sigma_intensity.restype = c_int
    L.sunny_geneig_launch_fourier_sigma.argtypes = [c_void_p, c_size, c_size, c_size, c_int, c_size, c_size,
                                                    c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_fourier_sigma.restype = c_int
    L.sunny_geneig_launch_fourier_sigma_intensity.argtypes = [c_void_p, c_size, c_size, c_size, c_int, c_size,
                                                              c_size, c_size, c_size, c_int, ctypes.c_double,
                                                              c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_fourier_sigma_intensity.restype = c_int
    p_int, p_size = ctypes.POINTER(c_int), ctypes.POINTER(c_size)
    L.sunny_geneig_uneven_create.argtypes = [c_int, p_int, p_int, p_int, c_int]
    L.sunny_geneig_uneven_create.restype = c_void_p
    L.sunny_geneig_uneven_launch.argtypes = [c_void_p, p_size, p_size, p_size, p_size, p_size, p_int, c_size]
    L.sunny_geneig_uneven_launch.restype = c_int
    L.sunny_geneig_uneven_destroy.argtypes = [c_void_p]
    L.sunny_geneig_uneven_destroy.restype = None
    L.sunny_geneig_uneven_shape.argtypes = [c_void_p, p_int, p_int, p_int]
    L.sunny_geneig_uneven_shape.restype = c_int
    for name in ("sunny_geneig_matrix_size", "sunny_geneig_batches_per_block", "sunny_geneig_block_dim_x",
                 "sunny_geneig_kernel_mode"):
        getattr(L, name).argtypes = [c_void_p]
        getattr(L, name).restype = c_int
    L.sunny_geneig_shared_mem_bytes.argtypes = [c_void_p]
    L.sunny_geneig_shared_mem_bytes.restype = c_uint
    L.sunny_geneig_last_error.argtypes = []
    L.sunny_geneig_last_error.restype = c_char_p
    L.sunny_geneig_path_name.argtypes = [c_void_p]
    L.sunny_geneig_path_name.restype = c_char_p
    L.sunny_geneig_regime_name.argtypes = [c_void_p]
    L.sunny_geneig_regime_name.restype = c_char_p
    L.sunny_geneig_launch_noalloc.argtypes = [c_int, c_size, c_size, c_size, c_size, c_size, c_int, c_size]
    L.sunny_geneig_launch_noalloc.restype = c_int
    L.sunny_geneig_selftest_reciprocal.argtypes = [c_size, c_size, c_int, c_size]
    L.sunny_geneig_selftest_reciprocal.restype = c_int
    L.sunny_geneig_max_matrix_size.argtypes = []
    L.sunny_geneig_max_matrix_size.restype = c_int
    _lib = L
    return L


def last_error() -> str:
    return load().sunny_geneig_last_error().decode()
