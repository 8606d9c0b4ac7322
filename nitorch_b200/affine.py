"""Affine sampling without a materialised grid.

nitorch's resize and reslice (nitorch/spatial/_grid.py:618-754, 860-914)
build a dense grid with affine_grid (:579-615) -- 12 bytes per output voxel
written and read back -- and pull through it.  Here the kernels compute the
coordinate A [sub; 1] of every output voxel from the matrix itself
(``pp_affine_pull`` / ``pp_affine_push`` / ``pp_affine_grad_matrix``).

`affine_pull(input, mat, shape, ...)` samples (N, C, *inshape) images at
the affine coordinates of a `shape` lattice; `affine_push` is its adjoint.
Both are differentiable with respect to the image and the first D rows of
the (N, D[+1], D+1) matrices.
"""
import ctypes

import torch

from . import _lib
from .grid import bound_to_nitorch, inter_to_nitorch
from .spatial import _On, _require_cuda, _workspace, _wsptr, get_deterministic

__all__ = ["affine_pull", "affine_push", "resize_pull"]


def _options(interpolation, bound, extrapolate):
    b = bound_to_nitorch(bound if isinstance(bound, (list, tuple)) else [bound], as_type="enum")
    o = inter_to_nitorch(interpolation if isinstance(interpolation, (list, tuple)) else [interpolation],
                         as_type="enum")
    return _lib.options([int(x) for x in b], [int(x) for x in o], int(extrapolate),
                        _lib.PP_DETERMINISTIC if get_deterministic() else 0)


def _matrix(mat, N, dim, dtype):
    """(N, D, D+1) matrices with contiguous rows, in the grid dtype."""
    gdt = torch.float64 if dtype == torch.float64 else torch.float32
    m = mat.to(gdt)
    if m.dim() == 2:
        m = m[None]
    m = m[..., :dim, :].reshape(-1, dim, dim + 1)
    if m.shape[0] == 1 and N > 1:
        m = m.expand(N, dim, dim + 1)
    return m.contiguous()


def _pull(input, mat, shape, interpolation, bound, extrapolate):
    _require_cuda(input)
    L = _lib.load()
    out = torch.empty((input.shape[0], input.shape[1], *shape), dtype=input.dtype, device=input.device)
    opt = _options(interpolation, bound, extrapolate)
    with _On(input):
        _lib.check(L.pp_affine_pull(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(mat)),
                                    ctypes.byref(_lib.desc(out)), ctypes.byref(opt), _lib.stream_of(input)))
    return out


def _push(input, mat, shape, interpolation, bound, extrapolate):
    _require_cuda(input)
    L = _lib.load()
    out = torch.empty((input.shape[0], input.shape[1], *shape), dtype=input.dtype, device=input.device)
    opt = _options(interpolation, bound, extrapolate)
    ws, nws = _workspace(out)
    with _On(input):
        _lib.check(L.pp_affine_push(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(mat)),
                                    ctypes.byref(_lib.desc(out)), ctypes.byref(opt), _lib.stream_of(input),
                                    _wsptr(ws), nws))
    return out


def _grad_matrix(grad, input, mat, interpolation, bound, extrapolate):
    """d <grad, pull(input; mat)> / d mat[:, :D], float32 (N, D, D+1)."""
    L = _lib.load()
    dim = mat.shape[-1] - 1
    if input.dtype == torch.float64:
        # the reduction is float32: run the float32 kernels on float64 data
        input, grad, mat = input.float(), grad.float(), mat.float()
    gm = torch.empty((input.shape[0], dim, dim + 1), dtype=torch.float32, device=input.device)
    nws = L.pp_affine_grad_workspace_bytes(ctypes.byref(_lib.desc(grad)))
    ws = torch.empty(nws, dtype=torch.uint8, device=input.device)
    opt = _options(interpolation, bound, extrapolate)
    with _On(input):
        _lib.check(L.pp_affine_grad_matrix(ctypes.byref(_lib.desc(grad)), ctypes.byref(_lib.desc(input)),
                                           ctypes.byref(_lib.desc(mat)), ctypes.byref(_lib.desc(gm)),
                                           ctypes.byref(opt), _lib.stream_of(input), _wsptr(ws), nws))
    return gm


def _unmatrix(g, mat_shape, dtype):
    """Gradient (N, D, D+1) back to the caller's matrix shape (zero rows for
    the homogeneous row, summed over a broadcast batch)."""
    dim = mat_shape[-1] - 1
    full = torch.zeros((g.shape[0], mat_shape[-2], dim + 1), dtype=dtype, device=g.device)
    full[:, :dim] = g
    if len(mat_shape) == 2:
        return full.sum(0)
    if mat_shape[0] == 1 and g.shape[0] > 1:
        full = full.sum(0, keepdim=True)
    return full.reshape(mat_shape)


class AffinePull(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, mat, shape, interpolation, bound, extrapolate):
        ctx.args = (tuple(input.shape[2:]), interpolation, bound, extrapolate)
        ctx.mat_info = (mat.shape, mat.dtype)
        m = _matrix(mat, input.shape[0], len(shape), input.dtype)
        ctx.save_for_backward(input, m)
        return _pull(input, m, shape, interpolation, bound, extrapolate)

    @staticmethod
    def backward(ctx, grad):
        input, m = ctx.saved_tensors
        inshape, interpolation, bound, extrapolate = ctx.args
        grad = grad.contiguous()
        gi = gm = None
        if ctx.needs_input_grad[0]:
            gi = _push(grad, m, inshape, interpolation, bound, extrapolate)
        if ctx.needs_input_grad[1]:
            g = _grad_matrix(grad, input, m, interpolation, bound, extrapolate)
            gm = _unmatrix(g, *ctx.mat_info)
        return gi, gm, None, None, None, None


class AffinePush(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, mat, shape, interpolation, bound, extrapolate):
        ctx.args = (tuple(input.shape[2:]), interpolation, bound, extrapolate)
        ctx.mat_info = (mat.shape, mat.dtype)
        m = _matrix(mat, input.shape[0], len(shape), input.dtype)
        ctx.save_for_backward(input, m)
        return _push(input, m, shape, interpolation, bound, extrapolate)

    @staticmethod
    def backward(ctx, grad):
        input, m = ctx.saved_tensors
        gshape, interpolation, bound, extrapolate = ctx.args
        grad = grad.contiguous()
        gi = gm = None
        if ctx.needs_input_grad[0]:
            gi = _pull(grad, m, gshape, interpolation, bound, extrapolate)
        if ctx.needs_input_grad[1]:
            # <g, push(y; A)> = <pull(g; A), y>: the matrix gradient of a pull of g against y
            g = _grad_matrix(input.contiguous(), grad, m, interpolation, bound, extrapolate)
            gm = _unmatrix(g, *ctx.mat_info)
        return gi, gm, None, None, None, None


def affine_pull(input, mat, shape, interpolation="linear", bound="zero", extrapolate=False):
    """Sample input (N, C, *inshape) at A [sub; 1] for every voxel `sub` of a
    `shape` lattice; mat (N|1, D[+1], D+1) or (D[+1], D+1)."""
    return AffinePull.apply(input, mat, tuple(int(s) for s in shape), interpolation, bound, extrapolate)


def affine_push(input, mat, shape, interpolation="linear", bound="zero", extrapolate=False):
    """Adjoint of affine_pull: splat input (N, C, *gridshape) into a `shape`
    lattice from the coordinates A [sub; 1]."""
    return AffinePush.apply(input, mat, tuple(int(s) for s in shape), interpolation, bound, extrapolate)


# --------------------------------------------------------------------- #
# diagonal maps (resize): separable kernel                              #
# --------------------------------------------------------------------- #

def resize_supported(input, interpolation):
    """pp_resize covers 3-D float32 / bfloat16 images with one B-spline order
    of at most 3 on every axis."""
    orders = inter_to_nitorch(interpolation if isinstance(interpolation, (list, tuple)) else [interpolation],
                              as_type="int")
    return (input.dim() == 5 and input.dtype in (torch.float32, torch.bfloat16) and input.is_cuda
            and len(set(orders)) == 1 and orders[0] <= 3)


def _resize(input, scales, shifts, shape, interpolation, bound, extrapolate):
    L = _lib.load()
    out = torch.empty((input.shape[0], input.shape[1], *shape), dtype=input.dtype, device=input.device)
    opt = _options(interpolation, bound, extrapolate)
    D3 = ctypes.c_double * 3
    with _On(input):
        _lib.check(L.pp_resize(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(out)),
                               D3(*[float(v) for v in scales]), D3(*[float(v) for v in shifts]),
                               ctypes.byref(opt), _lib.stream_of(input)))
    return out


def resize_status():
    """Device status word of the resize kernels (0: no bounded wait gave up)."""
    L = _lib.load()
    v = ctypes.c_uint32(0)
    _lib.check(L.pp_resize_status(ctypes.byref(v)))
    return int(v.value)


class ResizePull(torch.autograd.Function):
    """Sampling at x_d = scale_d o_d + shift_d (a diagonal affine map) by the
    separable kernel; the image gradient is the affine push of the same map."""

    @staticmethod
    def forward(ctx, input, scales, shifts, shape, interpolation, bound, extrapolate):
        ctx.args = (tuple(input.shape[2:]), tuple(scales), tuple(shifts), interpolation, bound, extrapolate)
        return _resize(input, scales, shifts, shape, interpolation, bound, extrapolate)

    @staticmethod
    def backward(ctx, grad):
        inshape, scales, shifts, interpolation, bound, extrapolate = ctx.args
        gi = None
        if ctx.needs_input_grad[0]:
            dim = len(scales)
            mat = torch.zeros((1, dim, dim + 1), dtype=torch.float32, device=grad.device)
            for d in range(dim):
                mat[0, d, d] = scales[d]
                mat[0, d, dim] = shifts[d]
            m = _matrix(mat, grad.shape[0], dim, grad.dtype)
            gi = _push(grad.contiguous(), m, inshape, interpolation, bound, extrapolate)
        return gi, None, None, None, None, None, None


def resize_pull(input, scales, shifts, shape, interpolation="linear", bound="zero", extrapolate=False):
    """Sample input (N, C, X, Y, Z) at x_d = scales[d] * o_d + shifts[d] for
    every voxel o of a `shape` lattice (pp_resize; positive scales)."""
    return ResizePull.apply(input, tuple(float(v) for v in scales), tuple(float(v) for v in shifts),
                            tuple(int(v) for v in shape), interpolation, bound, extrapolate)
