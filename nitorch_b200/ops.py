"""``torch.library`` operators over the C ABI.

The eight push/pull functions and the prefilter registered as PyTorch
custom operators (namespace ``nitorch_b200``), with fake (meta)
implementations for shape propagation and autograd formulas, so that they
compose with the dispatcher, ``torch.compile`` graphs and operator checks
like any ATen op:

    torch.ops.nitorch_b200.grid_pull(input, grid, bound, interpolation, extrapolate)

Arguments follow ``nitorch._C.spatial`` with integer codes for the bound and
the interpolation order (lists, one per axis, padded with the last entry).
The backward operators return every gradient (the drop-in module's
``requires_grad``-driven lists are a Python convention that custom
operators cannot express); the autograd formulas pass only what is needed.
"""
from typing import List, Tuple

import torch
from torch import Tensor

from . import coeff as _coeff
from . import spatial as _spatial
from .enums import BoundType, InterpolationType

__all__ = ["grid_pull", "grid_push", "grid_count", "grid_grad", "spline_coeff_nd"]


def _enums(bound, interpolation):
    return [BoundType(int(b)) for b in bound], [InterpolationType(int(i)) for i in interpolation]


def _with_grad(t, flag):
    return t.detach().requires_grad_(flag) if t.dtype.is_floating_point else t


# --------------------------------------------------------------------- #
# pull                                                                  #
# --------------------------------------------------------------------- #
@torch.library.custom_op("nitorch_b200::grid_pull", mutates_args=())
def grid_pull(input: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
              extrapolate: int) -> Tensor:
    return _spatial.grid_pull(input, grid, *_enums(bound, interpolation), extrapolate)


@grid_pull.register_fake
def _(input, grid, bound, interpolation, extrapolate):
    return input.new_empty((grid.shape[0], input.shape[1], *grid.shape[1:-1]))


@torch.library.custom_op("nitorch_b200::grid_pull_backward", mutates_args=())
def grid_pull_backward(grad: Tensor, input: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
                       extrapolate: int, need_input: bool, need_grid: bool) -> Tuple[Tensor, Tensor]:
    out = _spatial.grid_pull_backward(grad.contiguous(), _with_grad(input, need_input), _with_grad(grid, need_grid),
                                      *_enums(bound, interpolation), extrapolate)
    gi = out.pop(0) if need_input else input.new_zeros(input.shape)
    gg = out.pop(0) if need_grid else grid.new_zeros(grid.shape)
    return gi, gg


@grid_pull_backward.register_fake
def _(grad, input, grid, bound, interpolation, extrapolate, need_input, need_grid):
    return input.new_empty(input.shape), grid.new_empty(grid.shape)


def _pull_setup(ctx, inputs, output):
    input, grid, bound, interpolation, extrapolate = inputs
    ctx.save_for_backward(input, grid)
    ctx.opt = (bound, interpolation, extrapolate)


def _pull_bwd(ctx, grad):
    input, grid = ctx.saved_tensors
    gi, gg = torch.ops.nitorch_b200.grid_pull_backward(grad, input, grid, *ctx.opt, ctx.needs_input_grad[0],
                                                       ctx.needs_input_grad[1])
    return (gi if ctx.needs_input_grad[0] else None), (gg if ctx.needs_input_grad[1] else None), None, None, None


grid_pull.register_autograd(_pull_bwd, setup_context=_pull_setup)


# --------------------------------------------------------------------- #
# push                                                                  #
# --------------------------------------------------------------------- #
@torch.library.custom_op("nitorch_b200::grid_push", mutates_args=())
def grid_push(input: Tensor, grid: Tensor, shape: List[int], bound: List[int], interpolation: List[int],
              extrapolate: int) -> Tensor:
    return _spatial.grid_push(input, grid, shape, *_enums(bound, interpolation), extrapolate)


@grid_push.register_fake
def _(input, grid, shape, bound, interpolation, extrapolate):
    shape = list(shape) if len(shape) else list(input.shape[2:])
    return input.new_empty((grid.shape[0], input.shape[1], *shape))


@torch.library.custom_op("nitorch_b200::grid_push_backward", mutates_args=())
def grid_push_backward(grad: Tensor, input: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
                       extrapolate: int, need_input: bool, need_grid: bool) -> Tuple[Tensor, Tensor]:
    out = _spatial.grid_push_backward(grad.contiguous(), _with_grad(input, need_input), _with_grad(grid, need_grid),
                                      *_enums(bound, interpolation), extrapolate)
    gi = out.pop(0) if need_input else input.new_zeros(input.shape)
    gg = out.pop(0) if need_grid else grid.new_zeros(grid.shape)
    return gi, gg


@grid_push_backward.register_fake
def _(grad, input, grid, bound, interpolation, extrapolate, need_input, need_grid):
    return input.new_empty(input.shape), grid.new_empty(grid.shape)


def _push_setup(ctx, inputs, output):
    input, grid, shape, bound, interpolation, extrapolate = inputs
    ctx.save_for_backward(input, grid)
    ctx.opt = (bound, interpolation, extrapolate)


def _push_bwd(ctx, grad):
    input, grid = ctx.saved_tensors
    gi, gg = torch.ops.nitorch_b200.grid_push_backward(grad, input, grid, *ctx.opt, ctx.needs_input_grad[0],
                                                       ctx.needs_input_grad[1])
    return ((gi if ctx.needs_input_grad[0] else None), (gg if ctx.needs_input_grad[1] else None),
            None, None, None, None)


grid_push.register_autograd(_push_bwd, setup_context=_push_setup)


# --------------------------------------------------------------------- #
# count                                                                 #
# --------------------------------------------------------------------- #
@torch.library.custom_op("nitorch_b200::grid_count", mutates_args=())
def grid_count(grid: Tensor, shape: List[int], bound: List[int], interpolation: List[int],
               extrapolate: int) -> Tensor:
    return _spatial.grid_count(grid, shape, *_enums(bound, interpolation), extrapolate)


@grid_count.register_fake
def _(grid, shape, bound, interpolation, extrapolate):
    shape = list(shape) if len(shape) else list(grid.shape[1:-1])
    return grid.new_empty((grid.shape[0], 1, *shape))


@torch.library.custom_op("nitorch_b200::grid_count_backward", mutates_args=())
def grid_count_backward(grad: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
                        extrapolate: int) -> Tensor:
    return _spatial.grid_count_backward(grad.contiguous(), _with_grad(grid, True), *_enums(bound, interpolation),
                                        extrapolate)


@grid_count_backward.register_fake
def _(grad, grid, bound, interpolation, extrapolate):
    return grid.new_empty(grid.shape)


def _count_setup(ctx, inputs, output):
    grid, shape, bound, interpolation, extrapolate = inputs
    ctx.save_for_backward(grid)
    ctx.opt = (bound, interpolation, extrapolate)


def _count_bwd(ctx, grad):
    grid, = ctx.saved_tensors
    gg = torch.ops.nitorch_b200.grid_count_backward(grad, grid, *ctx.opt) if ctx.needs_input_grad[0] else None
    return gg, None, None, None, None


grid_count.register_autograd(_count_bwd, setup_context=_count_setup)


# --------------------------------------------------------------------- #
# spatial gradient                                                      #
# --------------------------------------------------------------------- #
@torch.library.custom_op("nitorch_b200::grid_grad", mutates_args=())
def grid_grad(input: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
              extrapolate: int) -> Tensor:
    return _spatial.grid_grad(input, grid, *_enums(bound, interpolation), extrapolate)


@grid_grad.register_fake
def _(input, grid, bound, interpolation, extrapolate):
    return input.new_empty((grid.shape[0], input.shape[1], *grid.shape[1:-1], grid.shape[-1]))


@torch.library.custom_op("nitorch_b200::grid_grad_backward", mutates_args=())
def grid_grad_backward(grad: Tensor, input: Tensor, grid: Tensor, bound: List[int], interpolation: List[int],
                       extrapolate: int, need_input: bool, need_grid: bool) -> Tuple[Tensor, Tensor]:
    out = _spatial.grid_grad_backward(grad.contiguous(), _with_grad(input, need_input), _with_grad(grid, need_grid),
                                      *_enums(bound, interpolation), extrapolate)
    gi = out.pop(0) if need_input else input.new_zeros(input.shape)
    gg = out.pop(0) if need_grid else grid.new_zeros(grid.shape)
    return gi, gg


@grid_grad_backward.register_fake
def _(grad, input, grid, bound, interpolation, extrapolate, need_input, need_grid):
    return input.new_empty(input.shape), grid.new_empty(grid.shape)


def _grad_setup(ctx, inputs, output):
    input, grid, bound, interpolation, extrapolate = inputs
    ctx.save_for_backward(input, grid)
    ctx.opt = (bound, interpolation, extrapolate)


def _grad_bwd(ctx, grad):
    input, grid = ctx.saved_tensors
    gi, gg = torch.ops.nitorch_b200.grid_grad_backward(grad, input, grid, *ctx.opt, ctx.needs_input_grad[0],
                                                       ctx.needs_input_grad[1])
    return (gi if ctx.needs_input_grad[0] else None), (gg if ctx.needs_input_grad[1] else None), None, None, None


grid_grad.register_autograd(_grad_bwd, setup_context=_grad_setup)


# --------------------------------------------------------------------- #
# prefilter                                                             #
# --------------------------------------------------------------------- #
@torch.library.custom_op("nitorch_b200::spline_coeff_nd", mutates_args=())
def spline_coeff_nd(input: Tensor, bound: List[int], order: List[int], dim: int) -> Tensor:
    """Prefilter codes of interpol.coeff (zero 0, replicate 1, dct1 2, dct2 3,
    dft 6); backward = forward, as nitorch's SplineCoeffND."""
    return _coeff.spline_coeff_nd(input, list(bound), list(order), dim, False)


@spline_coeff_nd.register_fake
def _(input, bound, order, dim):
    return input.new_empty(input.shape)


def _coeff_setup(ctx, inputs, output):
    _, bound, order, dim = inputs
    ctx.opt = (bound, order, dim)


def _coeff_bwd(ctx, grad):
    g = torch.ops.nitorch_b200.spline_coeff_nd(grad.contiguous(), *ctx.opt) if ctx.needs_input_grad[0] else None
    return g, None, None, None


spline_coeff_nd.register_autograd(_coeff_bwd, setup_context=_coeff_setup)
