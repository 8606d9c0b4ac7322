"""nitorch_b200: B200-native spline push/pull resampling.

A from-scratch CUDA (sm_100a) implementation of nitorch's compiled spline
push/pull path -- grid_pull, grid_push, grid_count, grid_grad and their
backward passes, B-spline orders 0-7, seven boundary conditions, 1/2/3-D --
plus the spline_coeff prefilter, behind a C ABI (include/nitorch_b200.h).

Entry points:
  nitorch_b200.grid_pull / grid_push / grid_count / grid_grad /
  spline_coeff / spline_coeff_nd / identity_grid   (nitorch.spatial API)
  nitorch_b200.pull_push    fused push(pull(.)) (normal operator), one pass
  nitorch_b200.grid_pull_grad  grid_pull and grid_grad of one input and grid, one pass
  nitorch_b200.resize / reslice / affine_pull / affine_push   affine sampling,
                            coordinates computed in the kernel (no grid)
  nitorch_b200.svf.exp      velocity exponentiation (scaling and squaring)
  nitorch_b200.grid_jacobian / grid_jacdet   Jacobians of transformation fields
  nitorch_b200.prolong / restrict            the multigrid solvers' resampling;
  nitorch_b200.multires     native fmg_prolongation / fmg_restriction, ni::resize
                            (modes, adjoint, normalisation) and their wrappers
  nitorch_b200.spatial      drop-in for the ``nitorch._C.spatial`` module
  nitorch_b200.ops          the same as torch.library operators (torch.ops.nitorch_b200.*)
  nitorch_b200.coeff        drop-in for ``interpol.coeff``
  nitorch_b200.batch        many uneven volumes in one persistent launch
  nitorch_b200.install()    route an installed nitorch through this backend
"""
from .api import (affine_grid, affine_pull, affine_push, grid_count, grid_grad, grid_pull, grid_pull_grad, grid_push,
                  identity_grid, pull_push, reslice, resize, spline_coeff, spline_coeff_nd)
from .enums import BoundType, GridAlignType, InterpolationType
from .jacobian import grid_jacdet, grid_jacobian
from .multires import fmg_prolongation, fmg_restriction, prolong, restrict
from .spatial import get_deterministic, set_deterministic
from . import spatial, coeff, grid, svf, ops, multires
from .integration import install

__all__ = ["grid_pull", "grid_push", "grid_count", "grid_grad", "grid_pull_grad", "pull_push", "affine_grid", "affine_pull",
           "affine_push", "resize", "reslice", "svf", "grid_jacobian", "grid_jacdet", "spline_coeff",
           "spline_coeff_nd", "identity_grid", "BoundType", "InterpolationType", "GridAlignType",
           "prolong", "restrict", "fmg_prolongation", "fmg_restriction", "multires",
           "set_deterministic", "get_deterministic", "spatial", "coeff", "grid",
           "install"]
