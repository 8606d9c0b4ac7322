"""Public spatial API: the ``nitorch.spatial`` push/pull entry points.

Same signatures, defaults, broadcasting and output shapes as
``nitorch/spatial/_grid.py``:
  grid_pull (146-205), grid_push (208-251), grid_count (254-287),
  grid_grad (290-328), spline_coeff (331-375), spline_coeff_nd (378-421),
  identity_grid (443-478); the broadcasting of leading dimensions and the
  label-map pull follow the behaviour of _grid.py:90-143 and 187-198.
"""
import torch

from .affine import affine_pull, affine_push, resize_pull, resize_supported
from .grid import GridCount, GridGrad, GridPull, GridPullGrad, GridPullPush, GridPush, SplineCoeff, SplineCoeffND


class _Layout:
    """How a caller's tensors fold into the kernels' layout and back.

    The kernels take images as (B, C, *spatial) and grids as (B, *spatial, D).
    Callers may add any number of leading batch dimensions to either tensor
    (broadcast against each other) and may leave the channel dimension out.
    ``lead`` holds the broadcast leading dimensions (flattened into B) and
    ``chan`` the channel dimensions the result gets back: the image's
    channel size when it has one, a singleton when it has none but there
    are leading dimensions, nothing otherwise."""

    __slots__ = ("lead", "chan", "dim")

    def __init__(self, lead, chan, dim):
        self.lead = tuple(lead)
        self.chan = tuple(chan)
        self.dim = dim

    def restore(self, out):
        """(B, C, *rest) kernel output -> (*lead, *chan, *rest)."""
        return out.reshape(*self.lead, *self.chan, *out.shape[2:])


def _fold(grid, image=None, shared_space=False):
    """Fold ``grid`` (*g_lead, *g_space, D) and ``image``
    (*i_lead, [C], *i_space) into kernel layout.  An image with exactly D
    dimensions has no channel; with more, dimension -D-1 is the channel.
    ``shared_space`` (push) broadcasts the two spatial shapes together as
    well.  Expanding can allocate when the reshape cannot view."""
    dim = grid.shape[-1]
    g_lead, g_space = grid.shape[:-dim - 1], grid.shape[-dim - 1:-1]
    if image is None:
        layout = _Layout(g_lead, (1,) if len(g_lead) else (), dim)
        return grid.reshape(-1, *g_space, dim), None, layout
    has_chan = image.dim() > dim
    nchan = image.shape[-dim - 1] if has_chan else 0
    i_lead = image.shape[:-dim - 1] if has_chan else ()
    i_space = image.shape[-dim:]
    if shared_space:
        g_space = i_space = torch.broadcast_shapes(g_space, i_space)
    lead = torch.broadcast_shapes(g_lead, i_lead)
    folded_grid = grid.expand(*lead, *g_space, dim).reshape(-1, *g_space, dim)
    folded_image = image.expand(*lead, nchan or 1, *i_space).reshape(-1, nchan or 1, *i_space)
    chan = (nchan,) if nchan else ((1,) if len(lead) else ())
    return folded_grid, folded_image, _Layout(lead, chan, dim)


def _pull_labels(labels, grid, interpolation, bound, extrapolate, prefilter):
    """Pull of an integer label map: every label is pulled as a 0/1 mask and
    each output voxel takes the label whose pulled mask is largest.  Masks
    are visited in increasing label order and a label must beat the best
    value so far strictly, so ties keep the smaller label and voxels where
    every mask pulls to zero (or less) get 0."""
    dim = grid.shape[-1]
    shape = (labels.shape[0], labels.shape[1], *grid.shape[1:-1])
    winner = labels.new_zeros(shape)
    score = grid.new_zeros(shape)
    for value in torch.unique(labels):
        mask = (labels == value).to(grid.dtype)
        if prefilter:
            mask = spline_coeff_nd(mask, interpolation=interpolation, bound=bound, dim=dim, inplace=True)
        prob = GridPull.apply(mask, grid, interpolation, bound, extrapolate)
        better = prob > score
        winner = torch.where(better, value.to(winner.dtype), winner)
        score = torch.maximum(score, prob)
    return winner


def grid_pull(input, grid, interpolation="linear", bound="zero", extrapolate=False,
              prefilter=False):
    """Sample an image at the voxel coordinates of `grid`.

    input: (..., [channel], *inshape); grid: (..., *outshape, dim)
    -> (..., [channel], *outshape).  Integer inputs are label maps (see
    _pull_labels).
    """
    grid, input, layout = _fold(grid, input)
    if not input.dtype.is_floating_point:
        return layout.restore(_pull_labels(input, grid, interpolation, bound, extrapolate, prefilter))
    if prefilter:
        input = spline_coeff_nd(input, interpolation=interpolation, bound=bound, dim=layout.dim)
    return layout.restore(GridPull.apply(input, grid, interpolation, bound, extrapolate))


def grid_push(input, grid, shape=None, interpolation="linear", bound="zero",
              extrapolate=False, prefilter=False):
    """Splat an image with respect to a deformation field (adjoint of pull).
    `shape` defaults to the image's own spatial shape; `prefilter` applies
    the spline prefilter to the splatted result."""
    grid, input, layout = _fold(grid, input, shared_space=True)
    target = tuple(input.shape[2:]) if shape is None else shape
    out = GridPush.apply(input, grid, target, interpolation, bound, extrapolate)
    if prefilter:
        out = spline_coeff_nd(out, interpolation=interpolation, bound=bound, dim=layout.dim, inplace=True)
    return layout.restore(out)


def pull_push(input, grid, interpolation="linear", bound="zero", extrapolate=False, prefilter=False):
    """push(pull(input, grid), grid) back onto the input's lattice, fused into
    one pass forward and one backward (the normal operator P^T P of a
    registration).  Equals grid_push(grid_pull(input, grid, ...), grid,
    input.shape[-dim:], ...) up to floating-point summation order; the grid
    may have any spatial shape.  `prefilter` applies to the pulled input, as
    in grid_pull.  Not in the reference, which runs the two calls."""
    grid, input, layout = _fold(grid, input)
    if prefilter:
        input = spline_coeff_nd(input, interpolation=interpolation, bound=bound, dim=layout.dim)
    return layout.restore(GridPullPush.apply(input, grid, interpolation, bound, extrapolate))


def grid_count(grid, shape=None, interpolation="linear", bound="zero", extrapolate=False):
    """Splatting weights of a deformation field (push of ones)."""
    grid, _, layout = _fold(grid)
    target = tuple(grid.shape[1:-1]) if shape is None else shape
    return layout.restore(GridCount.apply(grid, target, interpolation, bound, extrapolate))


def grid_grad(input, grid, interpolation="linear", bound="zero", extrapolate=False,
              prefilter=False):
    """Spatial gradients of the interpolant at the grid points:
    (..., [channel], *outshape, dim)."""
    grid, input, layout = _fold(grid, input)
    if prefilter:
        input = spline_coeff_nd(input, interpolation, bound, layout.dim)
    return layout.restore(GridGrad.apply(input, grid, interpolation, bound, extrapolate))


def grid_pull_grad(input, grid, interpolation="linear", bound="zero", extrapolate=False,
                   prefilter=False):
    """grid_pull and grid_grad of the same input and grid from one pass over
    each point's taps: ((..., [channel], *outshape), (..., [channel],
    *outshape, dim)), each equal to the separate call's result."""
    grid, input, layout = _fold(grid, input)
    if prefilter:
        input = spline_coeff_nd(input, interpolation, bound, layout.dim)
    pulled, grad = GridPullGrad.apply(input, grid, interpolation, bound, extrapolate)
    return layout.restore(pulled), layout.restore(grad)


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


def affine_grid(mat, shape):
    """Dense transformation grid (..., *shape, D) of affine matrices
    (..., D[+1], D+1) (nitorch/spatial/_grid.py:579-615).  resize / reslice
    below do not build it: their kernels compute the coordinates."""
    mat = torch.as_tensor(mat)
    shape = list(shape)
    dim = mat.shape[-1] - 1
    if dim != len(shape):
        raise ValueError(f"Dimension of the affine matrix ({dim}) and shape ({len(shape)}) are not the same.")
    if mat.shape[-2] not in (dim, dim + 1):
        raise ValueError(f"First argument should be matrices of shape (..., {dim}, {dim + 1}) or "
                         f"(..., {dim + 1}, {dim + 1}) but got {tuple(mat.shape)}.")
    batch = mat.shape[:-2]
    grid = identity_grid(shape, dtype=mat.dtype, device=mat.device)
    grid = grid.reshape([1] * len(batch) + list(grid.shape))
    lin = mat[..., :dim, :dim].reshape(*batch, *([1] * dim), dim, dim)
    off = mat[..., :dim, -1].reshape(*batch, *([1] * dim), dim)
    return torch.matmul(lin, grid[..., None])[..., 0] + off


def _resize_transform(inshape, factor, shape, anchor):
    """Output shape and per-axis (scale, shift) with input = scale * output
    + shift (nitorch/spatial/_grid.py:682-727)."""
    nb_dim = len(inshape)
    factor = list(factor) if isinstance(factor, (list, tuple)) else [factor or 0.] * nb_dim
    factor = (factor + factor[-1:] * nb_dim)[:nb_dim]
    factor = [f or 0. for f in factor]
    outshape = list(shape) if shape is not None else [None] * nb_dim
    outshape = (outshape + outshape[-1:] * nb_dim)[:nb_dim]
    anchor = [a[0].lower() for a in (anchor if isinstance(anchor, (list, tuple)) else [anchor] * nb_dim)]
    outshape = [o or max(1, int(i * f)) for i, o, f in zip(inshape, outshape, factor)]
    if any(not s for s in outshape):
        raise ValueError("Either factor or shape must be set in all dimensions")
    factor = [f or o / i for o, i, f in zip(outshape, inshape, factor)]
    scales, shifts = [], []
    for anch, f, i, o in zip(anchor, factor, inshape, outshape):
        if i == 1 or o == 1:
            anch = "e"
        if anch == "c":
            scales.append((i - 1) / (o - 1))
            shifts.append(0.)
        elif anch == "e":
            scale = i / o
            scales.append(scale)
            shifts.append(0.5 * (scale - 1))
        elif anch == "f":
            scales.append(1 / f)
            shifts.append(0.)
        elif anch == "l":
            scales.append(1 / f)
            shifts.append((i - 1) - (o - 1) / f)
        else:
            raise ValueError(f"Unknown anchor {anch}")
    return outshape, factor, scales, shifts


def resize(image, factor=None, shape=None, affine=None, anchor="c", dim=None, *args, **kwargs):
    """Resize an image by a factor or to a shape (nitorch/spatial/_grid.py:618-754):
    same arguments, anchors and output shapes; `prefilter` defaults to True.
    The sampling coordinates are computed in the kernel (no grid).  With
    `affine` (input orientation matrix, (..., D+1, D+1)), the resized
    image's orientation matrix is returned too."""
    image = torch.as_tensor(image)
    nb_dim = dim or (len(shape) if shape is not None else image.dim() - 2)
    inshape = list(image.shape[-nb_dim:])
    outshape, factor, scales, shifts = _resize_transform(inshape, factor, shape, anchor)
    interpolation = kwargs.pop("interpolation", args[0] if len(args) > 0 else "linear")
    bound = kwargs.pop("bound", args[1] if len(args) > 1 else "zero")
    extrapolate = kwargs.pop("extrapolate", args[2] if len(args) > 2 else False)
    prefilter = kwargs.pop("prefilter", True)
    batch = image.shape[:-nb_dim]
    x = image.reshape(-1, 1, *inshape)
    gdt = torch.float64 if x.dtype == torch.float64 else torch.float32
    mat = torch.zeros((nb_dim, nb_dim + 1), dtype=gdt, device=x.device)
    for d in range(nb_dim):
        mat[d, d] = scales[d]
        mat[d, nb_dim] = shifts[d]
    if prefilter:
        x = spline_coeff_nd(x, interpolation=interpolation, bound=bound, dim=nb_dim)
    if nb_dim == 3 and all(s > 0 for s in scales) and resize_supported(x, interpolation):
        # diagonal map: the separable kernel (equal to the affine pull)
        out = resize_pull(x, scales, shifts, outshape, interpolation, bound, extrapolate)
    else:
        out = affine_pull(x, mat, outshape, interpolation, bound, extrapolate)
    out = out.reshape(*batch, *outshape)
    if affine is not None:
        affine = torch.as_tensor(affine)
        T = torch.eye(nb_dim + 1, dtype=affine.dtype, device=affine.device)
        T[:nb_dim, :nb_dim] = torch.diag(torch.as_tensor(scales, dtype=affine.dtype, device=affine.device))
        T[:nb_dim, nb_dim] = torch.as_tensor(shifts, dtype=affine.dtype, device=affine.device)
        return out, affine.matmul(T)
    return out


def reslice(image, affine, affine_to, shape_to=None, **kwargs):
    """Reslice an image to another space (nitorch/spatial/_grid.py:860-914):
    the voxel-to-voxel matrix affine^-1 affine_to drives the kernel directly
    (no grid); `prefilter` defaults to True."""
    image = torch.as_tensor(image)
    gdt = torch.float64 if image.dtype == torch.float64 else torch.float32
    affine = torch.as_tensor(affine, dtype=gdt, device=image.device)
    affine_to = torch.as_tensor(affine_to, dtype=gdt, device=image.device)
    dim = affine.shape[-1] - 1
    batch = affine.shape[:-2]
    channels = image.shape[len(batch):-dim]
    shape = image.shape[-dim:]
    shape_to = list(shape_to or shape)
    transformation = torch.linalg.solve(affine, affine_to)
    n = 1
    for b in batch:
        n *= b
    nc = 1
    for c in channels:
        nc *= c
    x = image.reshape(n, nc, *shape)
    interpolation = kwargs.pop("interpolation", "linear")
    bound = kwargs.pop("bound", "zero")
    extrapolate = kwargs.pop("extrapolate", False)
    if kwargs.pop("prefilter", True):
        x = spline_coeff_nd(x, interpolation=interpolation, bound=bound, dim=dim)
    mat = transformation.reshape(-1, dim + 1, dim + 1)
    out = affine_pull(x, mat, shape_to, interpolation, bound, extrapolate)
    return out.reshape(*batch, *channels, *shape_to)
