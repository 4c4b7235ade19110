"""The C ABI library loads and behaves at its boundary without a GPU.

Mirrors the NULL-handle part of the reference's tests/common/test_c_api.cpp
(:86-117): accessors on NULL return -1 / 0 / "", destroy(NULL) is safe,
launch(NULL) returns INVALID_ARG with a non-empty last_error. No compute
call is made here.
"""
import ctypes
import re
import threading
from pathlib import Path

import pytest

from sunny_gen_eigensolver_b200 import _native as nat

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "sunny_geneig.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(sunny_geneig_[a-z_]+)\s*\(", text)))


def test_header_declarations_match_binding():
    assert declared_functions() == sorted(nat.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = nat.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_reference_abi_surface_present():
    # the eleven entry points of the reference's src/common/c_api.h:50-101
    ref = {"sunny_geneig_create", "sunny_geneig_create_ex", "sunny_geneig_destroy", "sunny_geneig_launch",
           "sunny_geneig_matrix_size", "sunny_geneig_batches_per_block", "sunny_geneig_block_dim_x",
           "sunny_geneig_shared_mem_bytes", "sunny_geneig_last_error", "sunny_geneig_path_name",
           "sunny_geneig_kernel_mode"}
    assert ref <= set(declared_functions())


def test_enum_values_match_reference():
    text = HEADER.read_text()
    for name, val in [("SUNNY_GENEIG_OK", 0), ("SUNNY_GENEIG_INVALID_ARG", -1), ("SUNNY_GENEIG_DEVICE_ERROR", -2),
                      ("SUNNY_GENEIG_COMPILE_ERROR", -3), ("SUNNY_GENEIG_LAUNCH_ERROR", -4),
                      ("SUNNY_GENEIG_CACHE_AUTO", 0), ("SUNNY_GENEIG_CACHE_NODISK", 1),
                      ("SUNNY_GENEIG_CACHE_NOCACHE", 2), ("SUNNY_GENEIG_TUNING_SUGGESTED", 0),
                      ("SUNNY_GENEIG_TUNING_AUTOTUNE", 1), ("SUNNY_GENEIG_KERNEL_UNIFIED", 0),
                      ("SUNNY_GENEIG_KERNEL_HYBRID", 1)]:
        m = re.search(rf"{name}\s*=\s*(-?\d+)", text)
        assert m and int(m.group(1)) == val, name


def test_null_handle_semantics():
    L = nat.load()
    assert L.sunny_geneig_matrix_size(None) == -1
    assert L.sunny_geneig_batches_per_block(None) == -1
    assert L.sunny_geneig_block_dim_x(None) == -1
    assert L.sunny_geneig_shared_mem_bytes(None) == 0
    assert L.sunny_geneig_path_name(None) == b""
    assert L.sunny_geneig_regime_name(None) == b""
    assert L.sunny_geneig_kernel_mode(None) == -1
    L.sunny_geneig_destroy(None)
    st = L.sunny_geneig_launch(None, 0, 0, 0, 0, 0, 8, 0)
    assert st == nat.STATUS_INVALID_ARG
    assert "NULL" in nat.last_error()
    assert L.sunny_geneig_max_matrix_size() >= 384


def test_last_error_is_thread_local():
    L = nat.load()
    L.sunny_geneig_launch(None, 0, 0, 0, 0, 0, 1, 0)
    assert nat.last_error() != ""
    seen = []
    t = threading.Thread(target=lambda: seen.append(nat.last_error()))
    t.start(); t.join()
    assert seen == [""]


def test_create_rejects_bad_size_before_touching_a_device():
    L = nat.load()
    for n in (0, -3, 100000):
        assert not L.sunny_geneig_create_ex(n, 0, 0, 0, 0, 0)
        assert "outside" in nat.last_error()


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = nat.load()
    assert not L.sunny_geneig_create(54, 0, 0, 0, 0)
    assert "CUDA" in nat.last_error() or "device" in nat.last_error()
