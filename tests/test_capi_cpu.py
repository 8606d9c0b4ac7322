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
    assert L.pp_abi_version() == 105
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
    # float32, 3-D, 2-4 channels: room for the channel-interleaved accumulator
    # of the vectorised push (optional: the push runs without it)
    d = _lib.desc(torch.zeros((1, 3, 8, 8, 8), dtype=torch.float32))
    assert L.pp_push_workspace_bytes(ctypes.byref(d), 0) == 8 * 8 * 8 * 4 * 4
    d = _lib.desc(torch.zeros((1, 1, 8, 8, 8), dtype=torch.float32))
    assert L.pp_push_workspace_bytes(ctypes.byref(d), 0) == 0
    d = _lib.desc(torch.zeros((1, 2, 8, 8), dtype=torch.float32))
    assert L.pp_push_workspace_bytes(ctypes.byref(d), 0) == 0


def test_regulariser_validation_on_host():
    """pp_regulariser / pp_regulariser_grid reject bad arguments before any
    CUDA call."""
    L = _lib.load()
    D3 = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    B3 = (ctypes.c_int32 * 3)(2, 2, 2)

    def field(x, out, w=None, h=None, bend=0.0):
        C = x.shape[1] if x.dim() > 1 else 1
        a = (ctypes.c_double * max(C, 1))(*([0.1] * max(C, 1)))
        b = (ctypes.c_double * max(C, 1))(*([bend] * max(C, 1)))
        return L.pp_regulariser(ctypes.byref(_lib.desc(x)), None if w is None else ctypes.byref(_lib.desc(w)),
                                None if h is None else ctypes.byref(_lib.desc(h)), ctypes.byref(_lib.desc(out)),
                                a, a, b, D3, B3, None)

    x = torch.zeros(1, 3, 4, 5, 6)
    assert field(torch.zeros(3, 4), torch.zeros(3, 4)) == _lib.PP_ERR_ARG  # no spatial dimension
    assert field(x.bfloat16(), x.bfloat16()) == _lib.PP_ERR_DTYPE  # float32 / float64 only
    assert field(torch.zeros(1, 65, 2, 2, 2), torch.zeros(1, 65, 2, 2, 2)) == _lib.PP_ERR_UNSUPPORTED
    assert field(x, torch.zeros(1, 3, 4, 5, 5)) == _lib.PP_ERR_ARG  # output shape
    assert field(x, x) == _lib.PP_ERR_ARG  # output overlaps the input
    assert field(x, torch.zeros_like(x), w=torch.ones_like(x), bend=1.0) == _lib.PP_ERR_UNSUPPORTED
    assert field(x, torch.zeros_like(x), h=torch.zeros(1, 4, 4, 5, 6)) == _lib.PP_ERR_ARG  # CC not 1/3/5/6
    g = torch.zeros(1, 4, 5, 6, 3)

    def grid(v, out, w=None, shear=0.0):
        return L.pp_regulariser_grid(ctypes.byref(_lib.desc(v)), None if w is None else ctypes.byref(_lib.desc(w)),
                                     None, ctypes.byref(_lib.desc(out)), 0.1, 1.0, 0.0, shear, 0.0, D3, B3, None)

    assert grid(torch.zeros(1, 4, 5, 6, 2), torch.zeros(1, 4, 5, 6, 2)) == _lib.PP_ERR_ARG  # D != dim
    assert grid(g, torch.zeros_like(g), w=torch.ones(1, 4, 5, 6), shear=1.0) == _lib.PP_ERR_UNSUPPORTED
    assert grid(g, torch.zeros_like(g), w=torch.ones(1, 4, 5, 7)) == _lib.PP_ERR_ARG


def test_svf_workspace_query():
    L = _lib.load()
    u = _lib.desc(torch.zeros((1, 4, 5, 6, 3), dtype=torch.float32))
    n = 4 * 5 * 6 * 3
    r = lambda b: (b + 255) // 256 * 256  # noqa: E731
    assert L.pp_svf_workspace_bytes(ctypes.byref(u), 0) == r(n // 3 * 16)
    assert L.pp_svf_workspace_bytes(ctypes.byref(u), _lib.PP_DETERMINISTIC) == 256 + r(n * 8) + r(n * 4)
    u2 = _lib.desc(torch.zeros((2, 7, 9, 2), dtype=torch.float64))
    assert L.pp_svf_workspace_bytes(ctypes.byref(u2), 0) == 0  # 2-D: scalar reductions, no workspace
    assert L.pp_svf_workspace_bytes(ctypes.byref(u2), _lib.PP_DETERMINISTIC) == 256 + r(2 * 7 * 9 * 2 * 8) * 2
    bad = _lib.desc(torch.zeros((1, 4, 5, 6, 2), dtype=torch.float32))  # 3-D field with 2 components
    assert L.pp_svf_workspace_bytes(ctypes.byref(bad), _lib.PP_DETERMINISTIC) == 0


def test_batch_plan_validation_on_host():
    """pp_batch_plan validates and plans on the host only (no CUDA call)."""
    from nitorch_b200.batch import _entry
    L = _lib.load()
    x = torch.zeros(1, 2, 6, 5, 4)
    g = torch.zeros(1, 6, 5, 4, 3)
    z = torch.zeros(1, 2, 6, 5, 4)
    w = torch.zeros(1, 2, 6, 5, 4)
    dx = torch.zeros(1, 2, 6, 5, 4)
    dg = torch.zeros(1, 6, 5, 4, 3)
    nb = L.pp_batch_plan_bytes(2)
    buf = ctypes.create_string_buffer(nb)
    p = ctypes.cast(buf, ctypes.c_void_p)

    def plan(mode, ents, nbytes=nb):
        arr = (_lib.PPBatchEntry * len(ents))(*ents)
        return L.pp_batch_plan(arr, len(ents), mode, 0, p, nbytes, None, 0)

    ok = _entry(src=x, grid=g, out=z, opt=_lib.options([2], [3], 0))
    assert plan(_lib.PP_BATCH_PULL_PUSH, [ok, ok]) == _lib.PP_OK
    bwd = _entry(src=x, trgt=w, grid=g, out=dx, gg=dg, opt=_lib.options([2], [1], 0))
    assert plan(_lib.PP_BATCH_PULL_PUSH_BACKWARD, [bwd, ok]) == _lib.PP_ERR_ARG  # second entry lacks trgt
    assert plan(_lib.PP_BATCH_PULL_PUSH_BACKWARD, [bwd]) == _lib.PP_OK
    assert plan(_lib.PP_BATCH_PULL_PUSH, [ok], nbytes=16) == _lib.PP_ERR_WORKSPACE
    high = _entry(src=x, grid=g, out=z, opt=_lib.options([2], [5], 0))
    assert plan(_lib.PP_BATCH_PULL_PUSH, [high]) == _lib.PP_ERR_UNSUPPORTED
    det = _entry(src=x, grid=g, out=z, opt=_lib.options([2], [1], 0, flags=_lib.PP_DETERMINISTIC))
    assert plan(_lib.PP_BATCH_PULL_PUSH, [det]) == _lib.PP_ERR_WORKSPACE  # the fixed-point scratch is required
    arr = (_lib.PPBatchEntry * 2)(det, ok)
    # header + int64 per output element, plus the interleaved accumulator of `ok`
    assert L.pp_batch_scratch_bytes(arr, 2, _lib.PP_BATCH_PULL_PUSH) == \
        256 + 2 * 6 * 5 * 4 * 8 // 256 * 256 + 256 + 6 * 5 * 4 * 2 * 4 // 256 * 256 + 256
    small = _entry(src=x, grid=g, out=torch.zeros(1, 2, 6, 5, 3), opt=_lib.options([2], [1], 0))
    assert plan(_lib.PP_BATCH_PULL_PUSH, [small]) == _lib.PP_ERR_ARG
    half = _entry(src=x, grid=g, out=z.bfloat16(), opt=_lib.options([2], [1], 0))
    assert plan(_lib.PP_BATCH_PULL_PUSH, [half]) == _lib.PP_ERR_DTYPE
    assert plan(3, [ok]) == _lib.PP_ERR_UNSUPPORTED  # count is not a batched mode
    assert L.pp_batch_run(None, None) == _lib.PP_ERR_ARG
    # interleaved scratch: 2-4 channel scatter entries at orders 2-3 only
    arr = (_lib.PPBatchEntry * 2)(ok, high)
    assert L.pp_batch_scratch_bytes(arr, 2, _lib.PP_BATCH_PULL_PUSH) == 6 * 5 * 4 * 2 * 4 // 256 * 256 + 256
    lin = _entry(src=x, grid=g, out=z, opt=_lib.options([2], [1], 0))
    arr = (_lib.PPBatchEntry * 1)(lin)
    assert L.pp_batch_scratch_bytes(arr, 1, _lib.PP_BATCH_PULL_PUSH) == 0
    assert L.pp_batch_scratch_bytes(arr, 1, _lib.PP_BATCH_PULL) == 0


def test_brick_order_geometry():
    """Brick counts and workspace of the brick-major order (host side only):
    ceil(size / brick) bricks per axis and batch item; 3-D grids only."""
    L = _lib.load()
    grid = _t((2, 5, 6, 7, 3))
    src = (ctypes.c_int64 * 3)(21, 22, 27)
    assert L.pp_brick_count(ctypes.byref(grid), src) == 2 * 6 * 6 * 5
    nkeys = 2 * 6 * 6 * 5 * 96
    assert L.pp_brick_order_workspace_bytes(ctypes.byref(grid), src) >= nkeys * 4 + 2 * 2 * 5 * 6 * 7 * 4
    g2 = _t((1, 5, 6, 2))
    assert L.pp_brick_count(ctypes.byref(g2), src) == -1
    assert b"3-D" in L.pp_last_error()
    rc = L.pp_brick_order(ctypes.byref(grid), src, None, None, None, None, 0, None)
    assert rc == _lib.PP_ERR_ARG
