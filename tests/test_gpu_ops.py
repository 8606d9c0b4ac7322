"""torch.library operators (nitorch_b200.ops): torch's operator checks
(schema, fake implementation, autograd registration), values against the
nitorch._C.spatial-compatible functions (identical calls, bit-identical
outputs) and gradcheck through the operators."""
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200.ops  # noqa: F401
from nitorch_b200 import spatial
from nitorch_b200.enums import BoundType, InterpolationType

pytestmark = pytest.mark.gpu

OPS = torch.ops.nitorch_b200


def _data(dtype=torch.float64, seed=0):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((1, 2, 5, 6, 4), generator=g, dtype=dtype).cuda()
    grid = (torch.rand((1, 4, 5, 3, 3), generator=g, dtype=dtype) * 5 - 0.5).cuda()
    return x, grid


def test_opcheck_all_operators():
    x, grid = _data()
    y = torch.randn((1, 2, 4, 5, 3), dtype=torch.float64).cuda()
    gg = torch.randn((1, 2, 4, 5, 3, 3), dtype=torch.float64).cuda()
    checks = ["test_schema", "test_faketensor", "test_autograd_registration"]
    torch.library.opcheck(OPS.grid_pull, (x, grid, [2], [3], 1), test_utils=checks)
    torch.library.opcheck(OPS.grid_push, (y, grid, [5, 6, 4], [2], [3], 1), test_utils=checks)
    torch.library.opcheck(OPS.grid_count, (grid, [5, 6, 4], [2], [1], 1), test_utils=checks)
    torch.library.opcheck(OPS.grid_grad, (x, grid, [2], [3], 1), test_utils=checks)
    torch.library.opcheck(OPS.grid_pull_backward, (y, x, grid, [2], [3], 1, True, True), test_utils=checks)
    torch.library.opcheck(OPS.grid_grad_backward, (gg, x, grid, [2], [3], 1, True, True), test_utils=checks)
    torch.library.opcheck(OPS.spline_coeff_nd, (x, [3], [3], 3), test_utils=checks)


def test_operators_equal_module_functions():
    x, grid = _data(torch.float32, seed=1)
    b, o = [BoundType.dct2], [InterpolationType.cubic]
    assert torch.equal(OPS.grid_pull(x, grid, [2], [3], 0), spatial.grid_pull(x, grid, b, o, 0))
    y = spatial.grid_pull(x, grid, b, o, 0)
    a = OPS.grid_push(y, grid, [5, 6, 4], [2], [3], 0)
    r = spatial.grid_push(y, grid, [5, 6, 4], b, o, 0)
    assert (a - r).abs().max().item() <= 1e-5 * r.abs().max().item()
    assert torch.equal(OPS.grid_grad(x, grid, [2], [3], 0), spatial.grid_grad(x, grid, b, o, 0))


def test_gradcheck_through_operators():
    x, grid = _data()
    x.requires_grad_(True)
    grid.requires_grad_(True)
    assert gradcheck(lambda a, g: OPS.grid_pull(a, g, [2], [3], 1), (x, grid), nondet_tol=1e-12)
    assert gradcheck(lambda a, g: OPS.grid_grad(a, g, [5], [2], 1), (x, grid), nondet_tol=1e-12)
    y = torch.randn((1, 2, 4, 5, 3), dtype=torch.float64).cuda().requires_grad_(True)
    assert gradcheck(lambda a, g: OPS.grid_push(a, g, [5, 6, 4], [2], [1], 1), (y, grid), nondet_tol=1e-12)
    assert gradcheck(lambda g: OPS.grid_count(g, [5, 6, 4], [2], [1], 1), (grid,), nondet_tol=1e-12)
