"""Jacobians and Jacobian determinants of transformation fields.

The counterparts of nitorch.spatial.grid_jacobian / grid_jacdet
(nitorch/spatial/_grid.py:917-1013).  Without `sample`, one kernel
(``pp_grid_jacobian``) takes central finite differences of the displacement
with the boundary condition (as nitorch's diff does,
nitorch/spatial/_finite_differences.py:32-222) and writes the D x D matrices
and / or their determinants -- the determinant alone never materialises the
matrices; its adjoint (``pp_grid_jacobian_backward``) makes both functions
differentiable.  With `sample`, the Jacobian is the spatial gradient of the
displacement at the sampled coordinates (grid_grad, linear) and the
determinant comes from ``pp_jacobian_det``.
"""
import ctypes

import torch

from . import _lib
from .grid import bound_to_nitorch
from .spatial import _On, _require_cuda

__all__ = ["grid_jacobian", "grid_jacdet"]


def _bound_code(bound):
    b = bound_to_nitorch(bound if isinstance(bound, (list, tuple)) else [bound], as_type="enum")
    return int(b[0])


def _vs(voxel_size, dim):
    v = list(voxel_size) if isinstance(voxel_size, (list, tuple)) else [voxel_size]
    v = [float(x) for x in (v + v[-1:] * dim)[:dim]]
    return (ctypes.c_double * 3)(*(v + [1.0] * (3 - dim)))


def _flat(field):
    dim = field.shape[-1]
    return field.reshape(-1, *field.shape[-dim - 1:])


def _jac_fd(field, want_jac, want_det, bound, vs, is_grid, add_identity):
    _require_cuda(field)
    L = _lib.load()
    f = _flat(field)
    dim = f.shape[-1]
    jac = torch.empty((*f.shape, dim), dtype=f.dtype, device=f.device) if want_jac else None
    det = torch.empty(f.shape[:-1], dtype=f.dtype, device=f.device) if want_det else None
    with _On(f):
        _lib.check(L.pp_grid_jacobian(ctypes.byref(_lib.desc(f)), _lib.ref(_lib.desc(jac)), _lib.ref(_lib.desc(det)),
                                      _bound_code(bound), _vs(vs, dim), int(is_grid), int(add_identity),
                                      _lib.stream_of(f)))
    lead = field.shape[:-dim - 1]
    if jac is not None:
        jac = jac.reshape(*lead, *jac.shape[1:])
    if det is not None:
        det = det.reshape(*lead, *det.shape[1:])
    return jac, det


class _JacobianFD(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, det_only, bound, vs, is_grid, add_identity):
        ctx.args = (det_only, bound, vs, is_grid, add_identity)
        ctx.save_for_backward(field)
        jac, det = _jac_fd(field, not det_only, det_only, bound, vs, is_grid, add_identity)
        return det if det_only else jac

    @staticmethod
    def backward(ctx, grad):
        field, = ctx.saved_tensors
        det_only, bound, vs, is_grid, add_identity = ctx.args
        L = _lib.load()
        f = _flat(field)
        dim = f.shape[-1]
        g = grad.reshape(f.shape[:-1]) if det_only else grad.reshape(*f.shape, dim)
        gf = torch.empty_like(f)
        gj, gd = (None, g) if det_only else (g, None)
        with _On(f):
            _lib.check(L.pp_grid_jacobian_backward(_lib.ref(_lib.desc(gj)), _lib.ref(_lib.desc(gd)),
                                                   ctypes.byref(_lib.desc(f)), ctypes.byref(_lib.desc(gf)),
                                                   _bound_code(bound), _vs(vs, dim), int(is_grid),
                                                   int(add_identity), _lib.stream_of(f)))
        return gf.reshape(field.shape), None, None, None, None, None


class _Det(torch.autograd.Function):
    @staticmethod
    def forward(ctx, jac):
        L = _lib.load()
        dim = jac.shape[-1]
        m = jac.reshape(-1, dim, dim)
        det = torch.empty(m.shape[0], dtype=jac.dtype, device=jac.device)
        with _On(m):
            _lib.check(L.pp_jacobian_det(ctypes.byref(_lib.desc(m)), ctypes.byref(_lib.desc(det)), None, None,
                                         _lib.stream_of(m)))
        ctx.save_for_backward(jac)
        return det.reshape(jac.shape[:-2])

    @staticmethod
    def backward(ctx, grad):
        jac, = ctx.saved_tensors
        L = _lib.load()
        dim = jac.shape[-1]
        m = jac.reshape(-1, dim, dim)
        g = grad.reshape(-1).contiguous()
        gj = torch.empty_like(m)
        with _On(m):
            _lib.check(L.pp_jacobian_det(ctypes.byref(_lib.desc(m)), None, ctypes.byref(_lib.desc(g)),
                                         ctypes.byref(_lib.desc(gj)), _lib.stream_of(m)))
        return gj.reshape(jac.shape)


def _sampled_jacobian(grid, sample, bound, type, add_identity, extrapolate):
    from .api import grid_grad
    dim = grid.shape[-1]
    if type == "grid":
        from .api import identity_grid
        grid = grid - identity_grid(grid.shape[-dim - 1:-1], dtype=grid.dtype, device=grid.device)
    jac = grid_grad(grid.movedim(-1, -dim - 1), sample, bound=bound, extrapolate=extrapolate)
    jac = jac.movedim(-dim - 2, -2)
    if add_identity:
        jac = jac + torch.eye(dim, dtype=jac.dtype, device=jac.device)
    return jac


def grid_jacobian(grid, sample=None, bound="dft", voxel_size=1, type="grid", add_identity=True,
                  extrapolate=True):
    """Jacobian (..., *spatial, dim, dim) of a transformation (type 'grid')
    or displacement ('disp') field (..., *spatial, dim); jac[..., i, j] =
    d psi_i / d x_j.  Same arguments as nitorch.spatial.grid_jacobian."""
    if type not in ("grid", "disp"):
        raise ValueError(f"unknown field type {type}")
    if sample is not None:
        return _sampled_jacobian(grid, sample, bound, type, add_identity, extrapolate)
    return _JacobianFD.apply(grid, False, bound, voxel_size, type == "grid", add_identity)


def grid_jacdet(grid, sample=None, bound="dft", voxel_size=1, type="grid", add_identity=True,
                extrapolate=True):
    """Determinant (..., *spatial) of grid_jacobian; without `sample` the
    matrices are never materialised."""
    if type not in ("grid", "disp"):
        raise ValueError(f"unknown field type {type}")
    if sample is not None:
        return _Det.apply(_sampled_jacobian(grid, sample, bound, type, add_identity, extrapolate))
    return _JacobianFD.apply(grid, True, bound, voxel_size, type == "grid", add_identity)
