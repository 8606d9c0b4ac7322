"""Stationary velocity fields: exponentiation by scaling and squaring.

The counterpart of ``nitorch.spatial.exp`` (nitorch/spatial/_svf.py:11-98):
the velocity is scaled by 2^-steps and composed with itself `steps` times,
    u <- u + u o (id + u)
(_svf.py:85-94; the pull of _pull_vel, :323-362: dft bound, linear order,
extrapolation on by default).  Each squaring is ONE kernel
(``pp_svf_compose``: the identity is added on the fly, no grid is
materialised, the add is fused into the pull), and the backward pass is the
exact adjoint of every composition in reverse, one kernel each
(``pp_svf_compose_backward``: push of the gradient, grid gradient and the
identity term in one pass).  The reference differentiates the same
composition chain with autograd (its default; ``anagrad`` selects an
approximate analytic backward there, which is not reproduced: the argument
is accepted and the exact gradient is returned).

Fields are ([batch], *spatial, dim) float32 / float64 CUDA tensors,
displacement components last, dim 1-3.
"""
import ctypes

import torch

from . import _lib
from .grid import bound_to_nitorch, inter_to_nitorch
from .spatial import _On, _require_cuda, get_deterministic

__all__ = ["exp", "compose", "compose_backward"]


def _options(interpolation, bound, extrapolate=True, flags=0):
    b = bound_to_nitorch(bound if isinstance(bound, (list, tuple)) else [bound], as_type="enum")
    o = inter_to_nitorch(interpolation if isinstance(interpolation, (list, tuple)) else [interpolation],
                         as_type="enum")
    return _lib.options([int(x) for x in b], [int(x) for x in o], int(extrapolate), flags)


def _batched(field):
    dim = field.shape[-1]
    if field.dim() == dim + 1:
        return field[None], True
    return field.reshape(-1, *field.shape[-dim - 1:]), False


def _field_like(u):
    """An empty field shaped like u ([batch], *spatial, dim).  3-D float32
    fields are the first three slots of a four-slot buffer: 16-byte voxels,
    one load or store each in the composition kernels."""
    if u.dtype == torch.float32 and u.shape[-1] == 3 and u.dim() in (4, 5):
        return torch.empty(*u.shape[:-1], 4, dtype=u.dtype, device=u.device)[..., :3]
    return torch.empty(u.shape, dtype=u.dtype, device=u.device)


def compose(disp, interpolation="linear", bound="dft", extrapolate=True):
    """u + pull(u, id + u) for a displacement field u ([batch], *spatial, dim)."""
    _require_cuda(disp)
    L = _lib.load()
    u, unbatched = _batched(disp)
    out = _field_like(u)
    opt = _options(interpolation, bound, extrapolate)
    with _On(u):
        _lib.check(L.pp_svf_compose(ctypes.byref(_lib.desc(u)), ctypes.byref(_lib.desc(out)), ctypes.byref(opt),
                                    _lib.stream_of(u)))
    return out[0] if unbatched else out.reshape(disp.shape)


def compose_backward(grad, disp, interpolation="linear", bound="dft", extrapolate=True, deterministic=None):
    """Gradient of <grad, compose(disp)> with respect to disp.  With
    `deterministic` (default: the library's deterministic switch,
    ``set_deterministic``) the result is bit-identical from run to run."""
    _require_cuda(disp)
    L = _lib.load()
    u, unbatched = _batched(disp)
    g = grad.reshape(u.shape)
    det = get_deterministic() if deterministic is None else bool(deterministic)
    flags = _lib.PP_DETERMINISTIC if det else 0
    opt = _options(interpolation, bound, extrapolate, flags)
    du = _lib.desc(u)
    nws = L.pp_svf_workspace_bytes(ctypes.byref(du), flags)
    # the vector-reduction accumulator, or the fixed-point accumulator and the
    # per-voxel terms of the deterministic mode
    ws = torch.empty(nws, dtype=torch.uint8, device=u.device) if nws else None
    if ws is not None and not det:
        # the result is the accumulator's first three slots (no copy)
        out = ws[:u.numel() // 3 * 16].view(torch.float32).view(*u.shape[:-1], 4)[..., :3]
    else:
        out = torch.empty(u.shape, dtype=u.dtype, device=u.device)
    with _On(u):
        _lib.check(L.pp_svf_compose_backward(ctypes.byref(_lib.desc(g)), ctypes.byref(du),
                                             ctypes.byref(_lib.desc(out)), ctypes.byref(opt), _lib.stream_of(u),
                                             None if ws is None else ctypes.c_void_p(ws.data_ptr()), nws))
    return out[0] if unbatched else out.reshape(disp.shape)


_IDENTITY = {}


def _identity(shape, dtype, device):
    """The identity grid (*shape, dim), built once per (shape, dtype, device)
    and kept (read only) for later calls."""
    key = (tuple(shape), dtype, str(device))
    ident = _IDENTITY.get(key)
    if ident is None:
        mesh = torch.meshgrid(*[torch.arange(s, dtype=dtype, device=device) for s in shape], indexing="ij")
        ident = torch.stack(mesh, dim=-1)
        if len(_IDENTITY) >= 8:
            _IDENTITY.clear()
        _IDENTITY[key] = ident
    return ident


class _Exp(torch.autograd.Function):

    @staticmethod
    def forward(ctx, vel, inverse, steps, interpolation, bound, displacement):
        scale = (-1.0 if inverse else 1.0) / (2 ** steps)
        if steps:
            u = torch.mul(vel, scale, out=_field_like(vel))  # in the compositions' layout
        else:
            u = vel * scale
        states = []
        for _ in range(steps):
            states.append(u)
            u = compose(u, interpolation, bound)
        ctx.save_for_backward(*states)
        ctx.args = (inverse, steps, interpolation, bound)
        if not displacement:
            dim = vel.shape[-1]
            u = u + _identity(vel.shape[-dim - 1:-1], vel.dtype, vel.device)
        return u

    @staticmethod
    def backward(ctx, grad):
        inverse, steps, interpolation, bound = ctx.args
        states = ctx.saved_tensors
        g = grad.contiguous()
        for u in reversed(states):
            g = compose_backward(g, u, interpolation, bound)
        g = g / (2 ** steps)
        if inverse:
            g = -g
        return g, None, None, None, None, None


def exp(vel, inverse=False, steps=8, interpolation="linear", bound="dft", displacement=False, anagrad=False):
    """Exponentiate a stationary velocity field by scaling and squaring.

    vel: ([batch], *spatial, dim) velocity; returns the transformation
    (identity + displacement) or, with `displacement`, the displacement.
    Same arguments as nitorch.spatial.exp; gradients are exact (see the
    module docstring for `anagrad`)."""
    if steps < 0:
        raise ValueError("steps must be non-negative")
    return _Exp.apply(vel, inverse, int(steps), interpolation, bound, displacement)
