"""Public spatial API: the ``nitorch.spatial`` push/pull entry points.

Same signatures, defaults, broadcasting and output shapes as
``nitorch/spatial/_grid.py``:
  grid_pull (146-205), grid_push (208-251), grid_count (254-287),
  grid_grad (290-328), spline_coeff (331-375), spline_coeff_nd (378-421),
  identity_grid (443-478), with the pre/post-processing of _preproc /
  _postproc (90-143) and the soft label-map pull (187-198).
"""
import torch

from .grid import GridCount, GridGrad, GridPull, GridPullPush, GridPush, SplineCoeff, SplineCoeffND


def _expanded_shape(*shapes):
    return list(torch.broadcast_shapes(*[tuple(s) for s in shapes]))


def _preproc(grid, input=None, mode=None):
    """Broadcast and reshape to (B, C, *spatial) / (B, *spatial, D)
    (_grid.py:90-127).  This *can* allocate (expand + reshape)."""
    dim = grid.shape[-1]
    if input is None:
        spatial = grid.shape[-dim - 1:-1]
        batch = grid.shape[:-dim - 1]
        grid = grid.reshape([-1, *spatial, dim])
        info = dict(batch=batch, channel=[1] if batch else [], dim=dim)
        return grid, info

    grid_spatial = grid.shape[-dim - 1:-1]
    grid_batch = grid.shape[:-dim - 1]
    input_spatial = input.shape[-dim:]
    channel = 0 if input.dim() == dim else input.shape[-dim - 1]
    input_batch = input.shape[:-dim - 1]

    if mode == "push":
        grid_spatial = input_spatial = _expanded_shape(grid_spatial, input_spatial)

    batch = _expanded_shape(grid_batch, input_batch)
    grid = grid.expand([*batch, *grid_spatial, dim])
    grid = grid.reshape([-1, *grid_spatial, dim])
    input = input.expand([*batch, channel or 1, *input_spatial])
    input = input.reshape([-1, channel or 1, *input_spatial])

    out_channel = [channel] if channel else ([1] if batch else [])
    info = dict(batch=batch, channel=out_channel, dim=dim)
    return grid, input, info


def _postproc(out, shape_info, mode):
    dim = shape_info["dim"]
    if mode != "grad":
        spatial = out.shape[-dim:]
        feat = []
    else:
        spatial = out.shape[-dim - 1:-1]
        feat = [out.shape[-1]]
    batch = shape_info["batch"]
    channel = shape_info["channel"]
    return out.reshape([*batch, *channel, *spatial, *feat])


def grid_pull(input, grid, interpolation="linear", bound="zero", extrapolate=False,
              prefilter=False):
    """Sample an image at the voxel coordinates of `grid`.

    input: (..., [channel], *inshape); grid: (..., *outshape, dim)
    -> (..., [channel], *outshape).  Integer inputs are label maps: each
    label is pulled as a soft mask and the arg-max label is returned.
    """
    grid, input, shape_info = _preproc(grid, input)
    batch, channel = input.shape[:2]
    dim = grid.shape[-1]

    if not input.dtype.is_floating_point:
        out = input.new_zeros([batch, channel, *grid.shape[1:-1]])
        pmax = grid.new_zeros([batch, channel, *grid.shape[1:-1]])
        for label in input.unique():
            soft = (input == label).to(grid.dtype)
            if prefilter:
                soft = spline_coeff_nd(soft, interpolation=interpolation, bound=bound,
                                       dim=dim, inplace=True)
            soft = GridPull.apply(soft, grid, interpolation, bound, extrapolate)
            out[soft > pmax] = label
            pmax = torch.max(pmax, soft)
    else:
        if prefilter:
            input = spline_coeff_nd(input, interpolation=interpolation, bound=bound, dim=dim)
        out = GridPull.apply(input, grid, interpolation, bound, extrapolate)
    return _postproc(out, shape_info, mode="pull")


def grid_push(input, grid, shape=None, interpolation="linear", bound="zero",
              extrapolate=False, prefilter=False):
    """Splat an image with respect to a deformation field (adjoint of pull)."""
    grid, input, shape_info = _preproc(grid, input, mode="push")
    dim = grid.shape[-1]
    if shape is None:
        shape = tuple(input.shape[2:])
    out = GridPush.apply(input, grid, shape, interpolation, bound, extrapolate)
    if prefilter:
        out = spline_coeff_nd(out, interpolation=interpolation, bound=bound, dim=dim,
                              inplace=True)
    return _postproc(out, shape_info, mode="push")


def pull_push(input, grid, interpolation="linear", bound="zero", extrapolate=False, prefilter=False):
    """push(pull(input, grid), grid) back onto the input's lattice, fused into
    one pass forward and one backward (the normal operator P^T P of a
    registration).  Equals grid_push(grid_pull(input, grid, ...), grid,
    input.shape[-dim:], ...) up to floating-point summation order; the grid
    may have any spatial shape.  `prefilter` applies to the pulled input, as
    in grid_pull.  Not in the reference, which runs the two calls."""
    grid, input, shape_info = _preproc(grid, input)
    dim = grid.shape[-1]
    if prefilter:
        input = spline_coeff_nd(input, interpolation=interpolation, bound=bound, dim=dim)
    out = GridPullPush.apply(input, grid, interpolation, bound, extrapolate)
    return _postproc(out, shape_info, mode="push")


def grid_count(grid, shape=None, interpolation="linear", bound="zero", extrapolate=False):
    """Splatting weights of a deformation field (push of ones)."""
    grid, shape_info = _preproc(grid)
    if shape is None:
        shape = tuple(grid.shape[1:-1])
    out = GridCount.apply(grid, shape, interpolation, bound, extrapolate)
    return _postproc(out, shape_info, mode="count")


def grid_grad(input, grid, interpolation="linear", bound="zero", extrapolate=False,
              prefilter=False):
    """Spatial gradients of the interpolant at the grid points:
    (..., [channel], *outshape, dim)."""
    grid, input, shape_info = _preproc(grid, input)
    dim = grid.shape[-1]
    if prefilter:
        input = spline_coeff_nd(input, interpolation, bound, dim)
    out = GridGrad.apply(input, grid, interpolation, bound, extrapolate)
    return _postproc(out, shape_info, mode="grad")


def spline_coeff(input, interpolation="linear", bound="dct2", dim=-1, inplace=False):
    """Interpolating spline coefficients along one dimension."""
    return SplineCoeff.apply(input, bound, interpolation, dim, inplace)


def spline_coeff_nd(input, interpolation="linear", bound="dct2", dim=None, inplace=False):
    """Interpolating spline coefficients along the last `dim` dimensions."""
    return SplineCoeffND.apply(input, bound, interpolation, dim, inplace)


def identity_grid(shape, dtype=None, device=None):
    """Identity deformation field (*shape, dim) in voxel coordinates."""
    mesh1d = [torch.arange(float(s), dtype=dtype, device=device) for s in shape]
    grid = torch.meshgrid(*mesh1d, indexing="ij")
    return torch.stack(grid, dim=-1)
