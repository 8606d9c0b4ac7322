"""Affine sampling without a materialised grid (resize / reslice): the
on-the-fly coordinates against grid_pull / grid_push on the materialised
affine grid (same library, pinned to the oracle), the oracle itself, the
matrix gradient against the grid-gradient chain rule, gradcheck, and the
resize / reslice conventions of nitorch.spatial.  Tolerances: float64
1e-12 relative, float32 1e-5 (1e-4 for the matrix gradient, a sum over
all points)."""
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200 as nb
from nitorch_b200 import api
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu


def _mat(dim, N, seed, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    A = torch.eye(dim + 1, dtype=torch.float64).repeat(N, 1, 1)
    A[:, :dim, :dim] += 0.15 * torch.randn((N, dim, dim), generator=g, dtype=torch.float64)
    A[:, :dim, dim] = 2.0 * torch.randn((N, dim), generator=g, dtype=torch.float64)
    return A.to(dtype).cuda()


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [0, 1, 3, 5])
@pytest.mark.parametrize("bound", ["dct2", "zero", "dft"])
def test_affine_pull_push_equal_materialised_grid(dim, order, bound):
    g = torch.Generator().manual_seed(dim * 10 + order)
    ishape, oshape = (11, 9, 10)[:dim], (8, 12, 7)[:dim]
    x = torch.randn((2, 3, *ishape), generator=g, dtype=torch.float64).cuda()
    A = _mat(dim, 2, seed=order + dim)
    grid = api.affine_grid(A, oshape)
    for ex in (False, True):
        a = api.affine_pull(x, A, oshape, order, bound, ex)
        b = nb.grid_pull(x, grid, order, bound, ex)
        assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-12
        y = torch.randn((2, 3, *oshape), generator=g, dtype=torch.float64).cuda()
        c = api.affine_push(y, A, ishape, order, bound, ex)
        d = nb.grid_push(y, grid, ishape, order, bound, ex)
        assert relerr(c.cpu().numpy(), d.cpu().numpy()) < 1e-12
    code = {"dct2": 2, "zero": 7, "dft": 5}[bound]
    ref = O.grid_pull(x.cpu().numpy(), grid.cpu().numpy(), [code], [order], 0)
    assert relerr(api.affine_pull(x, A, oshape, order, bound).cpu().numpy(), ref) < 1e-12


def test_affine_float32_lane_split_push():
    """3-D cubic push of 3 channels goes through the lane-split vector
    kernel; compare with the materialised-grid push."""
    g = torch.Generator().manual_seed(3)
    x = torch.randn((1, 3, 30, 28, 26), generator=g).cuda()
    A = _mat(3, 1, seed=3, dtype=torch.float32)
    grid = api.affine_grid(A, (30, 28, 26))
    a = api.affine_push(x, A, (30, 28, 26), 3, "dct2")
    b = nb.grid_push(x, grid, (30, 28, 26), 3, "dct2")
    assert relerr(a.double().cpu().numpy(), b.double().cpu().numpy()) < 1e-5


@pytest.mark.parametrize("dim", [2, 3])
def test_affine_matrix_gradient(dim):
    g = torch.Generator().manual_seed(5 + dim)
    ishape, oshape = (12, 10, 9)[:dim], (9, 11, 8)[:dim]
    x = torch.randn((2, 2, *ishape), generator=g).cuda()
    A = _mat(dim, 2, seed=dim, dtype=torch.float32)
    w = torch.randn((2, 2, *oshape), generator=g).cuda()
    # chain rule through the materialised grid
    Ar = A.clone().requires_grad_(True)
    xr = x.clone().requires_grad_(True)
    (nb.grid_pull(xr, api.affine_grid(Ar, oshape), 3, "dct2") * w).sum().backward()
    # on-the-fly coordinates
    As = A.clone().requires_grad_(True)
    xs = x.clone().requires_grad_(True)
    (api.affine_pull(xs, As, oshape, 3, "dct2") * w).sum().backward()
    assert relerr(xs.grad.cpu().numpy(), xr.grad.cpu().numpy()) < 1e-5
    assert relerr(As.grad[:, :dim].cpu().numpy(), Ar.grad[:, :dim].cpu().numpy()) < 1e-4
    assert torch.all(As.grad[:, dim:] == 0)


def test_affine_gradcheck_input():
    g = torch.Generator().manual_seed(7)
    x = torch.randn((1, 2, 5, 4, 5), generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    A = _mat(3, 1, seed=7)
    assert gradcheck(lambda t: api.affine_pull(t, A, (4, 5, 4), 3, "dct2", True), (x,), nondet_tol=1e-12)


def _resize_grid(inshape, factor, anchor, dtype, device):
    """The resize sampling grid as nitorch/spatial/_grid.py:690-734 builds
    it (restated here for the test): per axis, coordinates of the output
    voxels in input voxels for the anchor."""
    lin = []
    for i in inshape:
        o = max(1, int(i * factor))
        a = anchor if (i > 1 and o > 1) else "e"
        if a == "c":
            lin.append(torch.linspace(0, i - 1, o, dtype=dtype, device=device))
        elif a == "e":
            scale = i / o
            lin.append(torch.arange(0., o, dtype=dtype, device=device) * scale + 0.5 * (scale - 1))
        elif a == "f":
            lin.append(torch.arange(0., o, dtype=dtype, device=device) / factor)
        else:
            lin.append(torch.arange(0., o, dtype=dtype, device=device) / factor + ((i - 1) - (o - 1) / factor))
    return torch.stack(torch.meshgrid(*lin, indexing="ij"), -1)


@pytest.mark.parametrize("anchor", ["c", "e", "f", "l"])
def test_resize_matches_grid_form(anchor):
    g = torch.Generator().manual_seed(11)
    x = torch.randn((1, 2, 13, 11, 9), generator=g, dtype=torch.float64).cuda()
    coef = nb.spline_coeff_nd(x, 3, "dct2", dim=3)
    for factor in (2.0, 0.5, 1.7):
        out = api.resize(x, factor=factor, anchor=anchor, interpolation=3, bound="dct2")
        grid = _resize_grid(x.shape[2:], factor, anchor, x.dtype, x.device)[None]
        ref = nb.grid_pull(coef, grid, 3, "dct2")
        assert out.shape == ref.shape
        assert relerr(out.cpu().numpy(), ref.cpu().numpy()) < 1e-11


def test_reslice_matches_grid_form():
    g = torch.Generator().manual_seed(12)
    x = torch.randn((1, 1, 12, 10, 14), generator=g, dtype=torch.float64).cuda()
    aff = torch.eye(4, dtype=torch.float64).cuda()
    aff[:3, :3] *= 1.5
    aff_to = _mat(3, 1, seed=12)[0]
    out = api.reslice(x, aff, aff_to, (9, 9, 9), interpolation=1, bound="zero")
    T = torch.linalg.solve(aff, aff_to)
    grid = api.affine_grid(T, (9, 9, 9))[None]
    ref = nb.grid_pull(nb.spline_coeff_nd(x, 1, "zero", dim=3), grid, 1, "zero")
    assert out.shape == (1, 1, 9, 9, 9)
    assert relerr(out.cpu().numpy(), ref.cpu().numpy()) < 1e-12
