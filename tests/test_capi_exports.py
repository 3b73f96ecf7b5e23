"""The C-ABI library loads and exports every symbol include/wspm.h declares (CPU; no compute)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wspm.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wspm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "wspm_picard_step" in syms and "wspm_krylov_solve" in syms and len(syms) >= 15


def test_library_exports_every_declared_symbol():
    from wspm_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.EXPORTED) == set(declared_symbols())


def test_host_only_entry_points():
    from wspm_b200._lib import lib
    assert lib.wspm_version().decode().startswith("wspm-b200")
    assert lib.wspm_status_string(1).decode() == "iteration cap reached"
    assert lib.wspm_krylov_workspace_doubles(1000, 0, 0) > 5 * 1000
    assert lib.wspm_krylov_workspace_doubles(1000, 2, 33) == -1        # restart > 32 unsupported
    assert lib.wspm_picard_workspace_doubles(1000, 1) > 0


def test_null_arguments_are_rejected_without_a_gpu():
    from wspm_b200 import _lib
    lib = _lib.lib
    assert lib.wspm_spmv_f64(None, None, None, None, None) == _lib.WSPM_BAD_ARG
    assert lib.wspm_picard_create(None, None) == _lib.WSPM_BAD_ARG
    pat = _lib.WspmPattern()
    assert lib.wspm_jacobi_dinv(ctypes.byref(pat), None, None, None) == _lib.WSPM_BAD_ARG
    assert lib.wspm_ensemble_step(None, None, None, 0, None) == _lib.WSPM_BAD_ARG
    assert lib.wspm_ensemble_workspace_doubles(0, 10) == 0
