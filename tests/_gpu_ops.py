"""Run the eight nitorch._C.spatial-compatible functions of the CUDA
product on numpy inputs (tests only)."""
import numpy as np
import torch

from nitorch_b200 import spatial
from nitorch_b200.enums import BoundType, InterpolationType


def enums(bound, order):
    b = [BoundType(x) for x in (bound if isinstance(bound, (list, tuple)) else [bound])]
    o = [InterpolationType(x) for x in (order if isinstance(order, (list, tuple)) else [order])]
    return b, o


def cu(a, dtype, rg=False, grid=False):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if grid and dtype in (torch.bfloat16, torch.float16):
        t = t.to(torch.float32)
    else:
        t = t.to(dtype)
    t = t.cuda()
    if rg:
        t.requires_grad_(True)
    return t


def np64(t):
    return t.detach().double().cpu().numpy()


def all_ops(vol, grid, tgt, gpush, gcount, ggrad, bound, order, ex=1, dtype=torch.float64):
    b, o = enums(bound, order)
    V, Gd, T = cu(vol, dtype), cu(grid, dtype, grid=True), cu(tgt, dtype)
    out = {}
    out["pull"] = np64(spatial.grid_pull(V, Gd, b, o, ex))
    out["sgrad"] = np64(spatial.grid_grad(V, Gd, b, o, ex))
    out["push"] = np64(spatial.grid_push(T, Gd, list(vol.shape[2:]), b, o, ex))
    out["count"] = np64(spatial.grid_count(Gd, list(vol.shape[2:]), b, o, ex))
    Vr, Gr, Tr = cu(vol, dtype, True), cu(grid, dtype, True, grid=True), cu(tgt, dtype, True)
    r = spatial.grid_pull_backward(T, Vr, Gr, b, o, ex)
    out["pullbwd_in"], out["pullbwd_grid"] = np64(r[0]), np64(r[1])
    r = spatial.grid_push_backward(cu(gpush, dtype), Tr, Gr, b, o, ex)
    out["pushbwd_in"], out["pushbwd_grid"] = np64(r[0]), np64(r[1])
    out["countbwd_grid"] = np64(spatial.grid_count_backward(cu(gcount, dtype), Gr, b, o, ex))
    r = spatial.grid_grad_backward(cu(ggrad, dtype), Vr, Gr, b, o, ex)
    out["gradbwd_in"], out["gradbwd_grid"] = np64(r[0]), np64(r[1])
    return out


def oracle_ops(vol, grid, tgt, gpush, gcount, ggrad, bound, order, ex=1):
    from oracle import oracle as O
    b, o = [bound], [order]
    out = {}
    out["pull"] = O.grid_pull(vol, grid, b, o, ex)
    out["sgrad"] = O.grid_grad(vol, grid, b, o, ex)
    out["push"] = O.grid_push(tgt, grid, vol.shape[2:], b, o, ex)
    out["count"] = O.grid_count(grid, vol.shape[2:], b, o, ex)
    out["pullbwd_in"], out["pullbwd_grid"] = O.grid_pull_backward(tgt, vol, grid, b, o, ex)
    out["pushbwd_in"], out["pushbwd_grid"] = O.grid_push_backward(gpush, tgt, grid, b, o, ex)
    out["countbwd_grid"] = O.grid_count_backward(gcount, grid, b, o, ex)
    out["gradbwd_in"], out["gradbwd_grid"] = O.grid_grad_backward(ggrad, vol, grid, b, o, ex)
    return out


def relerr(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if b.size == 0:
        return 0.0
    return float(np.abs(a - b).max()) / max(float(np.abs(b).max()), 1e-30)
