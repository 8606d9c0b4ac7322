"""pp_sample_order_noalloc: the sample ordering for callers that cannot
allocate device memory when they need it (for example a host runtime that
owns all device memory up front, or one under a fixed budget).  It works out
of a fixed scratch array compiled into the library instead of a caller
workspace.

Called through the C ABI, twice in a row (the scratch keeps the previous
call's contents, so the second call checks that the state it needs is
cleared), and compared with the allocating entry point pp_sample_order.
Within one source voxel the order is arbitrary (atomic ranks), so the
comparison is exact on what the ordering defines: the result is a
permutation, and the source-voxel key sequence it produces is identical.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from nitorch_b200 import _lib

pytestmark = pytest.mark.gpu


def _keys(grid, src):
    from tests._cases import sort_keys
    return sort_keys(grid[None], src)


def _grid(shape, src, seed):
    r = np.random.default_rng(seed)
    mesh = np.stack(np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij"), -1)
    scale = (np.array(src) - 1) / (np.array(shape) - 1)
    g = mesh * scale + 1.5 * r.standard_normal(mesh.shape)
    return g[None].astype(np.float32)


def _call_noalloc(L, grid, src):
    nvox = grid.numel() // 3
    perm = torch.full((nvox,), -1, dtype=torch.int32, device="cuda")
    s = (ctypes.c_int64 * 3)(*src)
    rc = L.pp_sample_order_noalloc(ctypes.byref(_lib.desc(grid)), s, ctypes.c_void_p(perm.data_ptr()),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, perm


def _call_alloc(L, grid, src):
    nvox = grid.numel() // 3
    s = (ctypes.c_int64 * 3)(*src)
    d = _lib.desc(grid)
    nbytes = L.pp_sample_order_workspace_bytes(ctypes.byref(d), s)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    perm = torch.full((nvox,), -1, dtype=torch.int32, device="cuda")
    rc = L.pp_sample_order(ctypes.byref(d), s, ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                           nbytes, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.pp_last_error()
    return perm


def test_noalloc_matches_workspace_entry_point_twice():
    L = _lib.load()
    cases = [((40, 36, 32), (44, 40, 36), 0), ((24, 30, 18), (20, 26, 30), 1)]
    for shape, src, seed in cases:          # two calls in a row, different sizes
        g = _grid(shape, src, seed)
        G = torch.from_numpy(g).cuda()
        ref = _call_alloc(L, G, src).cpu().numpy()
        rc, perm = _call_noalloc(L, G, src)
        assert rc == 0, L.pp_last_error()
        torch.cuda.synchronize()
        perm = perm.cpu().numpy()
        assert np.array_equal(np.sort(perm), np.arange(perm.size))
        key = _keys(g[0], src)
        assert np.array_equal(key[perm], key[ref])
        assert np.all(np.diff(key[perm]) >= 0)


def test_noalloc_rejects_requests_beyond_its_scratch():
    L = _lib.load()
    G = torch.zeros((1, 160, 160, 160, 3), dtype=torch.float32, device="cuda")   # 4.1 M points
    rc, _ = _call_noalloc(L, G, (160, 160, 160))
    assert rc == _lib.PP_ERR_WORKSPACE
    assert b"fixed scratch" in L.pp_last_error()
