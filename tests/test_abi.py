"""The C-ABI library loads on a machine without a GPU, exports every entry point
declared in include/edlut_b200.h, and fails loudly (an error code and a message,
no crash, no CPU fallback) when no GPU is present."""
import ctypes
import os
import re

import pytest

from edlut_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "edlut_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(eb_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "eb_ctx_create" in syms and "eb_run" in syms and len(syms) >= 25


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) <= bound, set(declared_symbols()) - bound


def test_no_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    L = _lib.load()
    h = ctypes.c_void_p()
    rc = L.eb_ctx_create(0, None, ctypes.byref(h))
    assert rc == -2  # EB_ERR_CUDA
    assert L.eb_last_error().decode()


def test_null_arguments_are_rejected():
    L = _lib.load()
    assert L.eb_run(None, 10) == -1
    assert L.eb_finalize(None, None) == -1
    assert L.eb_get_counters(None, None, None, None) == -1
