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


# Accepted spellings of each boundary condition (case-insensitive), keyed by
# the canonical name that is also the BoundType member name.
_BOUND_SPELLINGS = {
    "replicate": ("replicate", "repeat", "border", "nearest"),
    "zero": ("zero", "zeros", "constant"),
    "dct2": ("dct2", "reflect", "reflection", "neumann"),
    "dct1": ("dct1", "mirror"),
    "dft": ("dft", "wrap", "circular"),
    "dst2": ("dst2", "antireflect", "dirichlet"),
    "dst1": ("dst1", "antimirror"),
}
_BOUND_BY_SPELLING = {s: canon for canon, spellings in _BOUND_SPELLINGS.items() for s in spellings}


def _bound_name(b):
    """Canonical name of one boundary condition given as a BoundType member or
    any accepted spelling; anything else (integers included) is rejected."""
    if isinstance(b, BoundType):
        return b.name        # enum aliases resolve to the canonical member
    name = _BOUND_BY_SPELLING.get(b.lower()) if isinstance(b, str) else None
    if name is None:
        raise ValueError(f"Unknown boundary condition {b}")
    return name


def bound_to_nitorch(bound, as_type="str"):
    """Normalise boundary conditions (behaviour of nitorch/_C/grid.py:92-136).

    `bound` is one value or a list / tuple of values; the result has the same
    form.  as_type: "str" -> canonical names, "enum" -> BoundType members,
    "int" / int -> the prefilter's integer codes."""
    is_seq = isinstance(bound, (list, tuple))
    names = [_bound_name(b) for b in (bound if is_seq else (bound,))]
    if as_type in ("int", int):
        out = [TS_BOUND[BoundType[n]] for n in names]
    elif as_type == "enum":
        out = [BoundType[n] for n in names]
    else:
        out = names
    return type(bound)(out) if is_seq else out[0]


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


class GridPullGrad(torch.autograd.Function):
    """pull and grid_grad of one input at one grid, computed in one pass;
    the backward adds the two backward passes."""

    @staticmethod
    def forward(ctx, input, grid, interpolation, bound, extrapolate):
        opt = _opt(bound, interpolation, extrapolate)
        pulled, grad = _spatial.grid_pull_grad(input, grid, *opt)
        ctx.opt = opt
        ctx.save_for_backward(input, grid)
        return pulled, grad

    @staticmethod
    def backward(ctx, g_pull, g_grad):
        var = ctx.saved_tensors
        grad_input = grad_grid = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            for g, fn in ((g_pull, _spatial.grid_pull_backward), (g_grad, _spatial.grid_grad_backward)):
                if g is None:
                    continue
                gi, gg = _unpack(ctx, fn(g.contiguous(), *var, *ctx.opt))
                grad_input = gi if grad_input is None else grad_input + gi
                grad_grid = gg if grad_grid is None else grad_grid + gg
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
