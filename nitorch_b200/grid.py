"""Autograd functions of the push/pull path.

Mirror of ``nitorch/_C/grid.py:89-383``: name normalisation of bounds and
orders (``bound_to_nitorch`` / ``inter_to_nitorch``, grid.py:92-186) and the
``torch.autograd.Function`` wrappers GridPull / GridPush / GridCount /
GridGrad / SplineCoeff / SplineCoeffND with the same forward signatures,
saved tensors and backward unpacking by ``needs_input_grad``
(grid.py:192-383).  The hand-written adjoints are the CUDA kernels behind
``spatial.*_backward``: pull's input gradient is the push kernel and its
grid gradient the fused derivative gather, both in one launch.
"""
import torch

from . import coeff as _coeff
from . import spatial as _spatial
from .enums import TS_BOUND, BoundType, InterpolationType

COMPILED_BACKEND = "B200"


def make_list(x):
    if not isinstance(x, (list, tuple)):
        x = [x]
    return list(x)


def bound_to_nitorch(bound, as_type="str"):
    """Convert boundary type to niTorch's convention (grid.py:92-136)."""
    intype = type(bound)
    if not isinstance(bound, (list, tuple)):
        bound = [bound]
    obound = []
    for b in bound:
        b = b.lower() if isinstance(b, str) else b
        if b in ("replicate", "repeat", "border", "nearest", BoundType.replicate):
            obound.append("replicate")
        elif b in ("zero", "zeros", "constant", BoundType.zero):
            obound.append("zero")
        elif b in ("dct2", "reflect", "reflection", "neumann", BoundType.dct2):
            obound.append("dct2")
        elif b in ("dct1", "mirror", BoundType.dct1):
            obound.append("dct1")
        elif b in ("dft", "wrap", "circular", BoundType.dft):
            obound.append("dft")
        elif b in ("dst2", "antireflect", "dirichlet", BoundType.dst2):
            obound.append("dst2")
        elif b in ("dst1", "antimirror", BoundType.dst1):
            obound.append("dst1")
        else:
            raise ValueError(f"Unknown boundary condition {b}")
    if as_type in ("enum", "int", int):
        obound = [getattr(BoundType, b) for b in obound]
        if as_type in ("int", int):
            obound = [TS_BOUND[b] for b in obound]
    if issubclass(intype, (list, tuple)):
        obound = intype(obound)
    else:
        obound = obound[0]
    return obound


def inter_to_nitorch(inter, as_type="str"):
    """Convert interpolation order to NITorch's convention (grid.py:139-186)."""
    intype = type(inter)
    if not isinstance(inter, (list, tuple)):
        inter = [inter]
    ointer = []
    names = ("nearest", "linear", "quadratic", "cubic", "fourth", "fifth", "sixth", "seventh")
    for o in inter:
        o = o.lower() if isinstance(o, str) else o
        for k, name in enumerate(names):
            if o == k or o == name or o is InterpolationType(k):
                ointer.append(k)
                break
        else:
            raise ValueError(f"Unknown interpolation order {o}")
    if as_type in ("enum", "str", str):
        ointer = [InterpolationType(o) for o in ointer]
        if as_type in ("str", str):
            ointer = [o.name for o in ointer]
    if issubclass(intype, (list, tuple)):
        ointer = intype(ointer)
    else:
        ointer = ointer[0]
    return ointer


def _opt(bound, interpolation, extrapolate):
    bound = bound_to_nitorch(make_list(bound), as_type="enum")
    interpolation = inter_to_nitorch(make_list(interpolation), as_type="enum")
    return bound, interpolation, int(extrapolate)


def _unpack(ctx, grads):
    grad_input = grad_grid = None
    if ctx.needs_input_grad[0]:
        grad_input = grads[0]
        if ctx.needs_input_grad[1]:
            grad_grid = grads[1]
    elif ctx.needs_input_grad[1]:
        grad_grid = grads[0]
    return grad_input, grad_grid


class GridPull(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, grid, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        output = _spatial.grid_pull(input, grid, *opt)
        ctx.opt = opt
        ctx.save_for_backward(input, grid)
        return output

    @staticmethod
    def backward(ctx, grad):
        var = ctx.saved_tensors
        grads = _spatial.grid_pull_backward(grad, *var, *ctx.opt)
        grad_input, grad_grid = _unpack(ctx, grads)
        return grad_input, grad_grid, None, None, None


class GridPush(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, grid, shape, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        output = _spatial.grid_push(input, grid, shape, *opt)
        ctx.opt = opt
        ctx.save_for_backward(input, grid)
        return output

    @staticmethod
    def backward(ctx, grad):
        var = ctx.saved_tensors
        grads = _spatial.grid_push_backward(grad, *var, *ctx.opt)
        grad_input, grad_grid = _unpack(ctx, grads)
        return grad_input, grad_grid, None, None, None, None


class GridPullPush(torch.autograd.Function):
    """push(pull(input, grid), grid) as one op: one pass forward, one pass
    backward.  Not in the reference, where it is GridPull then GridPush."""

    @staticmethod
    def forward(ctx, input, grid, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        output = _spatial.grid_pull_push(input, grid, *opt)
        ctx.opt = opt
        ctx.save_for_backward(input, grid)
        return output

    @staticmethod
    def backward(ctx, grad):
        var = ctx.saved_tensors
        grads = _spatial.grid_pull_push_backward(grad, *var, *ctx.opt)
        grad_input, grad_grid = _unpack(ctx, grads)
        return grad_input, grad_grid, None, None, None


class GridCount(torch.autograd.Function):

    @staticmethod
    def forward(ctx, grid, shape, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        output = _spatial.grid_count(grid, shape, *opt)
        ctx.opt = opt
        ctx.save_for_backward(grid)
        return output

    @staticmethod
    def backward(ctx, grad):
        var = ctx.saved_tensors
        grad_grid = None
        if ctx.needs_input_grad[0]:
            grad_grid = _spatial.grid_count_backward(grad, *var, *ctx.opt)
        return grad_grid, None, None, None, None


class GridGrad(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, grid, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        output = _spatial.grid_grad(input, grid, *opt)
        ctx.opt = opt
        ctx.save_for_backward(input, grid)
        return output

    @staticmethod
    def backward(ctx, grad):
        var = ctx.saved_tensors
        grad_input = grad_grid = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            grads = _spatial.grid_grad_backward(grad, *var, *ctx.opt)
            grad_input, grad_grid = _unpack(ctx, grads)
        return grad_input, grad_grid, None, None, None


class SplineCoeff(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, bound, interpolation, dim, inplace):
        bound = bound_to_nitorch(bound, as_type="int")
        interpolation = inter_to_nitorch(interpolation, as_type="int")
        opt = (bound, interpolation, dim, inplace)
        output = _coeff.spline_coeff(input, *opt)
        if input.requires_grad:
            ctx.opt = opt
        return output

    @staticmethod
    def backward(ctx, grad):
        # symmetric filter -> backward == forward (grid.py:352-357)
        grad = _coeff.spline_coeff(grad, *ctx.opt[:-1], inplace=False)
        return [grad] + [None] * 4


class SplineCoeffND(torch.autograd.Function):

    @staticmethod
    def forward(ctx, input, bound, interpolation, dim, inplace):
        bound = bound_to_nitorch(make_list(bound), as_type="int")
        interpolation = inter_to_nitorch(make_list(interpolation), as_type="int")
        opt = (bound, interpolation, dim, inplace)
        output = _coeff.spline_coeff_nd(input, *opt)
        if input.requires_grad:
            ctx.opt = opt
        return output

    @staticmethod
    def backward(ctx, grad):
        grad = _coeff.spline_coeff_nd(grad, *ctx.opt[:-1], inplace=False)
        return grad, None, None, None, None
