"""Multigrid resampling and nitorch's native resize.

* ``fmg_prolongation`` / ``fmg_restriction`` -- nitorch's native multigrid
  operators (nitorch/_C/src/multires.h:10-19, multires.cpp:24-74,
  impl/multires_common.cpp:419-500 and 587-660): the output voxel centre
  maps to x = (o + 1/2) in / out - 1/2; prolongation is the quadratic
  B-spline at x, restriction weights the four nodes from floor(x) - 1 by the
  linear B-spline of width in / out.  Computed by the separable TMA-staged
  kernel (``pp_fmg_prolongation`` / ``pp_fmg_restriction``).
* ``resize`` / ``resize_backward`` / ``prolongation[_backward]`` /
  ``restriction[_backward]`` -- nitorch's native ``ni::resize`` family
  (nitorch/_C/src/resize.cpp:19-128, impl/resize_common.cpp:1488-1660): the
  pull of the source at a diagonal map of the target lattice (always
  extrapolating), its adjoint push, and the normalisation by the scales.
  The pull runs the separable kernel (``pp_resize``) for 3-D float32 /
  bfloat16 images with one order <= 3, else the affine pull; the push runs
  the affine push.
* ``c_resize`` / ``c_prolongation`` / ``c_restriction`` /
  ``c_prolongation_grid`` / ``c_restriction_grid`` -- the Python wrappers of
  nitorch/_C/resize.py:64-215.
* ``prolong`` / ``restrict`` -- the multigrid solvers' pull / push based
  operators (nitorch/spatial/_solvers.py:147-224).

Signatures, defaults and output shapes follow the reference.  Where the
reference misbehaves the deviation is stated at the function: its native
operators raise on 1-D / 2-D images (computed here), its grid wrappers scale
the channels by factors taken after moving the output back to channel-last
(reproduced here).
"""
import ctypes
import math

import torch

from . import _lib, affine
from .enums import BoundType, GridAlignType, InterpolationType
from .grid import bound_to_nitorch, inter_to_nitorch
from .spatial import _On, _require_cuda

__all__ = ["fmg_prolongation", "fmg_restriction", "resize", "resize_backward", "prolongation",
           "prolongation_backward", "restriction", "restriction_backward", "c_resize", "c_prolongation",
           "c_restriction", "c_prolongation_grid", "c_restriction_grid", "prolong", "restrict"]


def _list(v, n):
    v = list(v) if isinstance(v, (list, tuple)) else [v]
    return (v + v[-1:] * max(0, n - len(v)))[:n]


def _defined(t):
    return t is not None and t.numel() > 0


def _bound_codes(bound, dim, default=BoundType.dct2):
    b = list(bound) if isinstance(bound, (list, tuple)) else ([bound] if bound is not None else [])
    b = [BoundType(x) if type(x) is int else x for x in (b or [default])]
    return [int(x) for x in bound_to_nitorch(_list(b, dim), as_type="enum")]


def _order_codes(interpolation, dim, default):
    o = list(interpolation) if isinstance(interpolation, (list, tuple)) else (
        [interpolation] if interpolation is not None else [])
    o = o or [default]
    return [int(x) for x in inter_to_nitorch(_list(o, dim), as_type="enum")]


def _check(input, name="input"):
    if not torch.is_tensor(input) or input.dim() < 3 or input.dim() > 5:
        raise RuntimeError(f"(): expected {name} with 1 to 3 spatial dimensions (N, C, *spatial)")
    if input.numel() == 0:
        raise RuntimeError(f"(): expected a non-empty {name}")
    _require_cuda(input)


# --------------------------------------------------------------------- #
# native multigrid operators                                            #
# --------------------------------------------------------------------- #

def _as3d(t):
    """(N, C, *spatial) -> (N, C, X, Y, Z) view with trailing singleton axes."""
    while t.dim() < 5:
        t = t.unsqueeze(-1)
    return t


def _multires(input, output, bound, restrict):
    _check(input)
    if input.dtype not in (torch.float32, torch.bfloat16):
        raise RuntimeError("(): the multigrid kernels take float32 or bfloat16 images")
    dim = input.dim() - 2
    if _defined(output):
        if output.shape[:2] != input.shape[:2] or output.dim() != input.dim():
            raise RuntimeError("(): expected output (N, C, *shape) matching input (N, C, *inshape)")
        if output.dtype != input.dtype or output.device != input.device:
            raise RuntimeError("(): output dtype / device must match input")
        shape = list(output.shape[2:])
    else:
        shape = [int(math.ceil(s / 2.0)) if restrict else int(math.floor(2.0 * s)) for s in input.shape[2:]]
    codes = _bound_codes(bound, dim)
    # padded axes (1 -> 1 voxel) replicate: the operator is the identity there
    codes3 = codes + [int(BoundType.replicate)] * (3 - dim)
    out = torch.empty((*input.shape[:2], *shape), dtype=input.dtype, device=input.device)
    L = _lib.load()
    opt = _lib.options(codes3, [1], 1)
    fn = L.pp_fmg_restriction if restrict else L.pp_fmg_prolongation
    with _On(input):
        _lib.check(fn(ctypes.byref(_lib.desc(_as3d(input))), ctypes.byref(_lib.desc(_as3d(out))),
                      ctypes.byref(opt), _lib.stream_of(input)))
    if _defined(output):
        output.copy_(out)
        return output
    return out


def fmg_prolongation(input, output=None, bound=()):
    """Prolongation to the lattice of `output`, or floor(2 s) per axis
    (nitorch/_C/src/multires.cpp:24-48).  input (N, C, *spatial), 1-3
    spatial axes (the reference raises on 1-D / 2-D inputs); `bound` a list
    of BoundType, default dct2."""
    return _multires(input, output, bound, False)


def fmg_restriction(input, output=None, bound=()):
    """Restriction to the lattice of `output`, or ceil(s / 2) per axis
    (nitorch/_C/src/multires.cpp:50-74)."""
    return _multires(input, output, bound, True)


# --------------------------------------------------------------------- #
# native resize                                                         #
# --------------------------------------------------------------------- #

def _affine(factor, n_src, n_tgt, mode):
    """(shift, scale) of one axis (nitorch/_C/src/impl/resize_common.cpp:
    1547-1566): target voxel w reads source x = scale w + shift."""
    if mode == int(GridAlignType.edge):
        return 0.5 * (n_src / n_tgt - 1), n_src / n_tgt
    if mode == int(GridAlignType.center):
        if n_tgt == 1:
            raise RuntimeError("(): center alignment of a one-voxel axis is undefined")
        return 0.0, (n_src - 1) / (n_tgt - 1)
    if mode == int(GridAlignType.last):
        if n_tgt == 1:
            raise RuntimeError("(): last alignment of a one-voxel axis is undefined")
        return factor * (n_src - 1) / (n_tgt - 1), 1.0 / factor
    return 0.0, 1.0 / factor


def _mode_codes(mode, dim):
    m = list(mode) if isinstance(mode, (list, tuple)) else ([mode] if mode is not None else [])
    m = m or [GridAlignType.center]
    out = []
    for v in _list(m, dim):
        if isinstance(v, str):
            v = {"e": GridAlignType.edge, "c": GridAlignType.center, "f": GridAlignType.first,
                 "l": GridAlignType.last}[v[0].lower()]
        out.append(int(v))
    return out


def resize(input, output=None, factor=(), bound=(), interpolation=(), mode=(), do_adjoint=False,
           normalize=False):
    """nitorch's native resize (nitorch/_C/src/resize.cpp:19-60): sample the
    source -- `input`, or `output` when `do_adjoint` -- on the target lattice
    through the diagonal map of `mode` (edge / center / first / last,
    default center) and `factor` (default 1), always extrapolating; with
    `do_adjoint`, push `input` (the target) into the source lattice instead.
    The missing lattice is floor(source * factor) (pull) or
    ceil(target / factor) (push).  `normalize` multiplies by the product of
    the scales.  Defaults: dct2, linear."""
    _check(input)
    dim = input.dim() - 2
    if isinstance(factor, (int, float)):
        factor = [factor]
    f = [float(v) for v in _list(list(factor) if factor else [1.0], dim)]
    if do_adjoint:
        f = [1.0 / v for v in f]
    if do_adjoint:
        tgt_shape = list(input.shape[2:])
        src_shape = list(output.shape[2:]) if _defined(output) else [int(math.ceil(s * f[d]))
                                                                     for d, s in enumerate(tgt_shape)]
    else:
        src_shape = list(input.shape[2:])
        tgt_shape = list(output.shape[2:]) if _defined(output) else [int(math.floor(s * f[d]))
                                                                     for d, s in enumerate(src_shape)]
    modes = _mode_codes(mode, dim)
    aff = [_affine(f[d], float(src_shape[d]), float(tgt_shape[d]), modes[d]) for d in range(dim)]
    shifts = [a[0] for a in aff]
    scales = [a[1] for a in aff]
    orders = [InterpolationType(c) for c in _order_codes(interpolation, dim, InterpolationType.linear)]
    bounds = [BoundType(c) for c in _bound_codes(bound, dim)]
    if do_adjoint:
        mat = _diag(scales, shifts, input)
        out = affine.affine_push(input, mat, src_shape, orders, bounds, True)
    elif affine.resize_supported(input, orders) and all(s > 0 for s in scales):
        out = affine.resize_pull(input, scales, shifts, tgt_shape, orders, bounds, True)
    else:
        out = affine.affine_pull(input, _diag(scales, shifts, input), tgt_shape, orders, bounds, True)
    if normalize:
        out = out * math.prod(scales)
    if _defined(output):
        output.copy_(out)
        return output
    return out


def _diag(scales, shifts, like):
    dim = len(scales)
    mat = torch.zeros((1, dim, dim + 1), dtype=torch.float64, device=like.device)
    for d in range(dim):
        mat[0, d, d] = scales[d]
        mat[0, d, dim] = shifts[d]
    return mat


def resize_backward(grad, output=None, factor=(), bound=(), interpolation=(), mode=(), do_adjoint=False,
                    normalize=False):
    """The adjoint of `resize` (nitorch/_C/src/resize.cpp:89-102): resize
    with the inverse factors and the adjoint flag flipped."""
    f = list(factor) if isinstance(factor, (list, tuple)) else [factor]
    return resize(grad, output, [1.0 / float(v) for v in f] or [1.0], bound, interpolation, mode,
                  not do_adjoint, normalize)


def _lattice(output, name):
    if not _defined(output):
        raise RuntimeError(f"(): {name} needs the output lattice: pass `output`")
    return output


def prolongation(input, output=None, bound=(), interpolation=()):
    """Native prolongation (nitorch/_C/src/resize.cpp:63-74): resize at
    factor 1, edge alignment, quadratic by default, onto `output`'s
    lattice (the input's own when no output is given, as there)."""
    return resize(input, output, [1.0], bound, interpolation or [InterpolationType.quadratic],
                  [GridAlignType.edge], False, False)


def restriction(input, output=None, bound=(), interpolation=()):
    """Native restriction (resize.cpp:76-87): the adjoint resize at factor
    1, edge alignment, linear by default, normalised."""
    return resize(input, output, [1.0], bound, interpolation or [InterpolationType.linear],
                  [GridAlignType.edge], True, True)


def prolongation_backward(grad, output=None, bound=(), interpolation=()):
    """resize.cpp:104-115: the adjoint of `prolongation`."""
    return resize(grad, output, [1.0], bound, interpolation or [InterpolationType.quadratic],
                  [GridAlignType.edge], True, False)


def restriction_backward(grad, output=None, bound=(), interpolation=()):
    """resize.cpp:117-128: the adjoint of `restriction`."""
    return resize(grad, output, [1.0], bound, interpolation or [InterpolationType.linear],
                  [GridAlignType.edge], False, True)


# --------------------------------------------------------------------- #
# nitorch/_C/resize.py wrappers                                         #
# --------------------------------------------------------------------- #

def c_resize(input, factor=None, bound="dct2", interpolation=1, mode="center", shape=None, output=None,
             adjoint=False, normalize=False):
    """nitorch/_C/resize.py:64-97."""
    if output is None and shape:
        output = input.new_zeros([*input.shape[:2], *shape])
    if torch.is_tensor(factor):
        factor = factor.double().tolist()
    if not factor and not shape:
        raise ValueError("At least one of factor or shape must be provided")
    return resize(input, output, factor or [1.0], bound, interpolation, mode, adjoint, normalize)


def _factor_shape(input, factor, shape, restrict):
    dim = input.dim() - 2
    if shape:
        return list(shape)
    f = _list(factor, 3)
    if restrict:
        return [int(math.ceil(s / v)) for s, v in zip(input.shape[2:], f[:dim])]
    return [int((s * v) // 1) for s, v in zip(input.shape[2:], f[:dim])]


def c_prolongation(input, factor=2., bound="dct2", shape=None, output=None):
    """nitorch/_C/resize.py:99-124: fmg prolongation onto `output`, `shape`
    or floor(s * factor)."""
    if output is None:
        output = input.new_zeros([*input.shape[:2], *_factor_shape(input, factor, shape, False)])
    return fmg_prolongation(input, output, bound)


def c_restriction(input, factor=2., bound="dct2", shape=None, output=None):
    """nitorch/_C/resize.py:126-151: fmg restriction onto `output`, `shape`
    or ceil(s / factor)."""
    if output is None:
        output = input.new_zeros([*input.shape[:2], *_factor_shape(input, factor, shape, True)])
    return fmg_restriction(input, output, bound)


def _grid_form(fn, input, factor, bound, shape, hessian, output):
    """nitorch/_C/resize.py:153-215: (N, *spatial, D) displacement grids.
    The channels are scaled by out / in of the LAST `dim` axes of the
    channel-first input and of the channel-last output, as there (in 3-D:
    (Y'/X, Z'/Y, D/Z) rather than (X'/X, Y'/Y, Z'/Z)); with `hessian`,
    squares and cross products of those factors."""
    dim = input.shape[-1]
    inp = input.movedim(-1, 1)
    if output is not None:
        output = output.movedim(-1, 1)
    out = fn(inp, factor, bound, shape, output)
    out = out.movedim(1, -1)
    fac = [o / i for i, o in zip(inp.shape[-dim:], out.shape[-dim:])]
    if not hessian:
        for c in range(dim):
            out[..., c] *= fac[c]
    else:
        count = dim
        for c in range(dim):
            out[..., c] *= fac[c] ** 2
            for cc in range(c + 1, dim):
                out[..., count] *= fac[c] * fac[cc]
                count += 1
    return out


def c_prolongation_grid(input, factor=2., bound="dct2", shape=None, hessian=False, output=None):
    """nitorch/_C/resize.py:153-187."""
    return _grid_form(c_prolongation, input, factor, bound, shape, hessian, output)


def c_restriction_grid(input, factor=2., bound="dct2", shape=None, hessian=False, output=None):
    """nitorch/_C/resize.py:189-215."""
    return _grid_form(c_restriction, input, factor, bound, shape, hessian, output)


# --------------------------------------------------------------------- #
# multigrid solvers' prolong / restrict                                 #
# --------------------------------------------------------------------- #

def _edge_map(src, tgt):
    """Edge-aligned diagonal map of nitorch/spatial/_solvers.py:170-177:
    target voxel o reads source x = o src / tgt + (src / tgt - 1) / 2."""
    return [s / t for s, t in zip(src, tgt)], [0.5 * (s / t - 1) for s, t in zip(src, tgt)]


def _channel_first(x, dim):
    """(..., *spatial, K) -> (B, K, *spatial) and the leading shape."""
    lead = x.shape[:-dim - 1]
    y = x.movedim(-1, -dim - 1)
    return y.reshape(-1, *y.shape[-dim - 1:]), lead


def prolong(x, shape=None, bound="dct2", order=2, dim=None, grid=None):
    """nitorch/spatial/_solvers.py:147-181: x (..., *spatial, K) pulled at
    the edge-aligned map of the `shape` lattice (default 2 * spatial),
    extrapolating.  With `grid`, the pull through that grid."""
    from .api import grid_pull
    if not x.dtype.is_floating_point:
        x = x.to(torch.get_default_dtype())
    dim = dim or (x.dim() - 1)
    if grid is not None:
        y = grid_pull(x.movedim(-1, -dim - 1), grid, bound=bound, interpolation=order, extrapolate=True)
        return y.movedim(-dim - 1, -1)
    in_sp = list(x.shape[-dim - 1:-1])
    out_sp = list(shape) if shape else [2 * s for s in in_sp]
    y, lead = _channel_first(x, dim)
    scales, shifts = _edge_map(in_sp, out_sp)
    orders = [InterpolationType(c) for c in _order_codes(order, dim, InterpolationType.quadratic)]
    bounds = [BoundType(c) for c in _bound_codes(bound, dim)]
    if affine.resize_supported(y, orders):
        z = affine.resize_pull(y, scales, shifts, out_sp, orders, bounds, True)
    else:
        z = affine.affine_pull(y, _diag(scales, shifts, y), out_sp, orders, bounds, True)
    return z.reshape(*lead, *z.shape[1:]).movedim(-dim - 1, -1)


def restrict(x, shape=None, bound="dct2", order=1, dim=None, grid=None):
    """nitorch/spatial/_solvers.py:184-224: x (..., *spatial, K) pushed from
    the edge-aligned map onto the `shape` lattice (default ceil(spatial / 2)),
    extrapolating, times prod(shape) / prod(spatial).  With `grid`, the push
    through that grid."""
    from .api import grid_push
    if not x.dtype.is_floating_point:
        x = x.to(torch.get_default_dtype())
    dim = dim or (x.dim() - 1)
    out_sp = list(x.shape[-dim - 1:-1])
    in_sp = list(shape) if shape else [int(math.ceil(s / 2)) for s in out_sp]
    if grid is not None:
        y = grid_push(x.movedim(-1, -dim - 1), grid, in_sp, bound=bound, interpolation=order, extrapolate=True)
    else:
        y, lead = _channel_first(x, dim)
        scales, shifts = _edge_map(in_sp, out_sp)
        orders = [InterpolationType(c) for c in _order_codes(order, dim, InterpolationType.linear)]
        bounds = [BoundType(c) for c in _bound_codes(bound, dim)]
        z = affine.affine_push(y, _diag(scales, shifts, y), in_sp, orders, bounds, True)
        y = z.reshape(*lead, *z.shape[1:])
    y = y.movedim(-dim - 1, -1)
    return y * (math.prod(in_sp) / math.prod(out_sp))
