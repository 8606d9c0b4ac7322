"""Regularisers of the native solvers: out = (hessian + regulariser) @ input.

The counterparts of ``nitorch._C.solve.c_regulariser`` and
``c_regulariser_grid`` (nitorch/_C/solve.py:21-142), with the same
arguments, defaults and shape handling, on the CUDA kernel of
``pp_regulariser`` / ``pp_regulariser_grid`` (include/nitorch_b200.h).
``nitorch.spatial.regulariser`` / ``regulariser_grid``
(nitorch/spatial/_regularisers.py:1057, 1168) call these when the input
needs no gradient.

Where the reference is defective the behaviour here is the intended one: a
call with every penalty zero returns the Hessian product (zeros without
one) instead of hanging, and weights / Hessians are read per batch item.
"""
import ctypes

import torch

from . import _lib
from .grid import bound_to_nitorch
from .spatial import _On, _require_cuda

__all__ = ["c_regulariser", "c_regulariser_grid"]


def _make_list(x, n=None):
    """nitorch/_C/utils.py:4-10: a list, padded with its last entry to n."""
    if not isinstance(x, (list, tuple)):
        x = [x]
    x = list(x)
    if n and x:
        x = x + max(0, n - len(x)) * x[-1:]
    return x


def _vector(x, n=None):
    if torch.is_tensor(x):
        x = x.double().tolist()
    return [float(v) for v in _make_list(x, n)]


def _unfold3(v, default):
    v = list(v) or [default]
    return [float(v[min(i, len(v) - 1)]) for i in range(3)]


def _bounds(bound):
    b = bound_to_nitorch(_make_list(bound), as_type="enum")
    return (ctypes.c_int32 * 3)(*[int(x) for x in _unfold3([int(x) for x in b], 0)])


def _doubles(v):
    return (ctypes.c_double * len(v))(*v)


def c_regulariser(input, weight=None, hessian=None, dim=None, absolute=0, membrane=0, bending=0, factor=1,
                  voxel_size=1, bound="dct2", output=None):
    """output = (hessian + regulariser) @ input for a field.

    input (N, C, *shape); weight (N, C|1, *shape); hessian (N, CC, *shape)
    with CC in {1, C, 2C-1, C(C+1)/2}; absolute / membrane / bending /
    factor: [sequences of] float per channel; voxel_size and bound per axis;
    leading dimensions are added / removed around `dim` spatial ones as the
    reference does (nitorch/_C/solve.py:21-78)."""
    _require_cuda(input)
    L = _lib.load()
    pad_dim = 0
    if dim:
        pad_dim = dim + 2 - input.dim()
        while input.dim() < dim + 2:
            input = input.unsqueeze(0)
    if weight is not None:
        pad_dim = min(pad_dim, input.dim() - weight.dim())
        while weight.dim() < input.dim():
            weight = weight.unsqueeze(0)
        weight = weight.to(input.dtype).expand_as(input)
    if hessian is not None:
        pad_dim = min(pad_dim, input.dim() - hessian.dim())
        while hessian.dim() < input.dim():
            hessian = hessian.unsqueeze(0)
        hessian = hessian.to(input.dtype).expand((input.shape[0], hessian.shape[1]) + tuple(input.shape[2:]))
    C = input.shape[1]
    voxel_size = _vector(voxel_size) or [1.0]
    absolute = _vector(absolute, C) or [0.0] * C
    membrane = _vector(membrane, C) or [0.0] * C
    bending = _vector(bending, C) or [0.0] * C
    factor = _vector(factor, C) or [1.0] * C
    absolute = [a * f for a, f in zip(absolute, factor)]
    membrane = [m * f for m, f in zip(membrane, factor)]
    bending = [b * f for b, f in zip(bending, factor)]
    if any(bending) and weight is not None:
        raise ValueError("RLS only implemented for membrane or absolute")
    out = torch.empty_like(input) if output is None else output
    with _On(input):
        _lib.check(L.pp_regulariser(
            ctypes.byref(_lib.desc(input)), None if weight is None else ctypes.byref(_lib.desc(weight)),
            None if hessian is None else ctypes.byref(_lib.desc(hessian)), ctypes.byref(_lib.desc(out)),
            _doubles(absolute[:C]), _doubles(membrane[:C]), _doubles(bending[:C]),
            _doubles(_unfold3(voxel_size, 1.0)), _bounds(bound), _lib.stream_of(input)))
    for _ in range(pad_dim):
        out = out.squeeze(0)
    return out


def c_regulariser_grid(input, weight=None, hessian=None, absolute=0, membrane=0, bending=0, lame=0, factor=1,
                       voxel_size=1, bound="dft", output=None):
    """output = (hessian + regulariser) @ input for a displacement field.

    input (N, *shape, D); weight (N, *shape); hessian (N, *shape, DD) with DD
    in {1, D, D(D+1)/2}; absolute, membrane, bending: float; lame: (shear,
    div); all scaled by `factor` (nitorch/_C/solve.py:80-142)."""
    _require_cuda(input)
    L = _lib.load()
    dim = input.shape[-1]
    pad_dim = dim + 2 - input.dim()
    while input.dim() < dim + 2:
        input = input.unsqueeze(0)
    if weight is not None:
        pad_dim = min(pad_dim, dim + 1 - weight.dim())
        while weight.dim() < dim + 1:
            weight = weight.unsqueeze(0)
        weight = weight.to(input.dtype).expand(input.shape[:-1])
    if hessian is not None:
        pad_dim = min(pad_dim, dim + 2 - hessian.dim())
        while hessian.dim() < input.dim():
            hessian = hessian.unsqueeze(0)
        hessian = hessian.to(input.dtype).expand(tuple(input.shape[:-1]) + (hessian.shape[-1],))
    voxel_size = _vector(voxel_size) or [1.0]
    absolute = float(absolute * factor)
    membrane = float(membrane * factor)
    bending = float(bending * factor)
    shear, div = (_make_list(lame, 2) or [0.0, 0.0])[:2]
    shear, div = float(shear * factor), float(div * factor)
    if (bending or shear or div) and weight is not None:
        raise ValueError("RLS only implemented for membrane or absolute")
    if output is None:
        out = torch.empty_like(input)
    else:
        out = output
        while out.dim() < input.dim():
            out = out.unsqueeze(0)
    with _On(input):
        _lib.check(L.pp_regulariser_grid(
            ctypes.byref(_lib.desc(input)), None if weight is None else ctypes.byref(_lib.desc(weight)),
            None if hessian is None else ctypes.byref(_lib.desc(hessian)), ctypes.byref(_lib.desc(out)),
            absolute, membrane, bending, shear, div, _doubles(_unfold3(voxel_size, 1.0)), _bounds(bound),
            _lib.stream_of(input)))
    for _ in range(pad_dim):
        out = out.squeeze(0)
    return out
