"""C-ABI library: loads, exports every symbol include/nitorch_b200.h
declares, and validates arguments on the host (no GPU needed: every call
here fails validation before any CUDA call)."""
import ctypes
import os
import re

import pytest
import torch

from nitorch_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "nitorch_b200.h")


def declared():
    src = open(HDR).read()
    return re.findall(r"PP_API\s+[\w\s\*]+?\b(pp_\w+)\s*\(", src)


def test_header_declares_exports():
    names = declared()
    assert len(names) >= 13
    assert set(names) == set(_lib.EXPORTS)


def test_library_exports_every_symbol():
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name), name
    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    for name in declared():
        assert re.search(rf"\bT {name}\b", out), name


def test_abi_version_and_error_state():
    L = _lib.load()
    assert L.pp_abi_version() == 100
    assert isinstance(L.pp_last_error(), bytes)


def _t(shape, dtype=torch.float32):
    return _lib.desc(torch.zeros(shape, dtype=dtype))


def test_validation_errors():
    L = _lib.load()
    opt = _lib.options([2], [3], 0)
    inp, grid, out = _t((1, 1, 4, 4, 4)), _t((1, 4, 4, 4, 2)), _t((1, 1, 4, 4, 4))
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(grid), ctypes.byref(out), ctypes.byref(opt), None)
    assert rc == _lib.PP_ERR_ARG
    assert b"expected grid to have size 3 in last dimension" in L.pp_last_error()
    grid = _t((1, 4, 4, 4, 3), torch.float64)
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(grid), ctypes.byref(out), ctypes.byref(opt), None)
    assert rc == _lib.PP_ERR_DTYPE
    grid = _t((1, 4, 4, 4, 3))
    bad = _lib.options([2], [9], 0)
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(grid), ctypes.byref(out), ctypes.byref(bad), None)
    assert rc == _lib.PP_ERR_ARG and b"order" in L.pp_last_error()
    bad = _lib.options([6], [1], 0)    # 'sliding' is not a push/pull bound
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(grid), ctypes.byref(out), ctypes.byref(bad), None)
    assert rc == _lib.PP_ERR_ARG
    wrong = _t((1, 2, 4, 4, 4))
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(grid), ctypes.byref(wrong), ctypes.byref(opt), None)
    assert rc == _lib.PP_ERR_ARG
    empty = _t((1, 4, 0, 4, 3))
    rc = L.pp_grid_pull(ctypes.byref(inp), ctypes.byref(empty), ctypes.byref(out), ctypes.byref(opt), None)
    assert rc == _lib.PP_ERR_ARG and b"non-empty" in L.pp_last_error()
    rc = L.pp_grid_pull(None, ctypes.byref(grid), ctypes.byref(out), ctypes.byref(opt), None)
    assert rc == _lib.PP_ERR_ARG and b"undefined" in L.pp_last_error()


def test_coeff_validation():
    L = _lib.load()
    a, b = _t((3, 5)), _t((3, 6))
    assert L.pp_spline_coeff(ctypes.byref(a), ctypes.byref(b), 3, 3, -1, None) == _lib.PP_ERR_ARG
    assert L.pp_spline_coeff(ctypes.byref(a), ctypes.byref(a), 3, 3, 5, None) == _lib.PP_ERR_ARG
    assert L.pp_spline_coeff(ctypes.byref(a), ctypes.byref(a), 3, 8, -1, None) == _lib.PP_ERR_ARG


def test_workspace_query():
    L = _lib.load()
    d = _lib.desc(torch.zeros((1, 2, 8, 8, 8), dtype=torch.bfloat16))
    n = L.pp_push_workspace_bytes(ctypes.byref(d), 0)
    assert n >= 2 * 8 * 8 * 8 * 4 and n % 256 == 0
    d = _lib.desc(torch.zeros((1, 2, 8, 8, 8), dtype=torch.float32))
    assert L.pp_push_workspace_bytes(ctypes.byref(d), 0) == 0
