"""Autograd of the CUDA product: the reference's gradcheck suite
(nitorch/tests/test_gradcheck_spatial.py: double, size 3 per dim, all
bounds and orders, 1/2/3-D, extrapolate=True) run on the GPU with torch's
default (strict) tolerances instead of the reference's rtol=1, plus the
grid_grad gradcheck that the reference leaves disabled ("FIXME") because of
its defects D2/D3, adjoint identities, and central finite differences of a
config-2 style pull -> push chain with the prefilter on a 24^3 crop."""
import numpy as np
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200 as nb
from nitorch_b200.enums import BoundType, InterpolationType

pytestmark = pytest.mark.gpu

BOUNDS = sorted(set(BoundType.__members__.values()), key=int)
ORDERS = sorted(set(InterpolationType.__members__.values()), key=int)


def make_data(shape, dtype=torch.double, seed=0):
    g = torch.Generator().manual_seed(seed)
    idg = nb.identity_grid(shape, dtype=dtype)[None]
    grid = idg + torch.randn(idg.shape, generator=g, dtype=dtype)
    vol = torch.randn((1, 1) + shape, generator=g, dtype=dtype)
    return vol.cuda(), grid.cuda()


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bound", BOUNDS)
@pytest.mark.parametrize("interpolation", ORDERS)
def test_gradcheck_pull_push_count_grad(dim, bound, interpolation):
    shape = (3,) * dim
    vol, grid = make_data(shape, seed=int(bound) * 10 + int(interpolation) + 100 * dim)
    vol.requires_grad_(True)
    grid.requires_grad_(True)
    assert gradcheck(nb.grid_pull, (vol, grid, interpolation, bound, True))
    assert gradcheck(nb.grid_push, (vol, grid, shape, interpolation, bound, True))
    assert gradcheck(nb.grid_count, (grid, shape, interpolation, bound, True))
    assert gradcheck(nb.grid_grad, (vol, grid, interpolation, bound, True))


@pytest.mark.parametrize("order", range(8))
@pytest.mark.parametrize("bound", ["replicate", "dct1", "dct2", "dst1", "dst2", "dft", "zero"])
def test_adjoint_pull_push(order, bound):
    torch.manual_seed(order)
    x = torch.randn(1, 2, 11, 12, 13, dtype=torch.double, device="cuda")
    grid = nb.identity_grid((9, 10, 8), dtype=torch.double, device="cuda")[None] * 1.2 - 1
    grid = grid + torch.randn_like(grid)
    y = torch.randn(1, 2, 9, 10, 8, dtype=torch.double, device="cuda")
    for ex in (False, True):
        a = (nb.grid_pull(x, grid, order, bound, ex) * y).sum()
        b = (x * nb.grid_push(y, grid, x.shape[2:], order, bound, ex)).sum()
        assert abs((a - b).item()) <= 1e-12 * abs(a.item())


def test_grid_grad_is_derivative_of_pull():
    torch.manual_seed(0)
    x = torch.randn(1, 2, 10, 11, 12, dtype=torch.double, device="cuda")
    grid = nb.identity_grid((6, 7, 8), dtype=torch.double, device="cuda")[None] + 1.3
    grid = grid + 0.5 * torch.randn_like(grid)
    for order in (2, 3, 5, 7):
        gg = nb.grid_grad(x, grid, order, "dct2", True)
        eps = 1e-6
        for d in range(3):
            e = torch.zeros_like(grid)
            e[..., d] = eps
            fd = (nb.grid_pull(x, grid + e, order, "dct2", True)
                  - nb.grid_pull(x, grid - e, order, "dct2", True)) / (2 * eps)
            assert torch.allclose(gg[..., d], fd, rtol=1e-6, atol=1e-7)


def test_config2_crop_finite_differences():
    """prefilter -> pull -> push chain, order 3, dct2, on a 24^3 crop of a
    config-2 style input; autograd gradient vs central FD (float64)."""
    from nitorch_b200 import workloads
    torch.manual_seed(0)
    x, grid = workloads.config2(size=24, channels=3, disp_std=2.0)
    x, grid = x.cuda(), grid.cuda()
    w = torch.randn(1, 3, 24, 24, 24, dtype=torch.double, device="cuda")

    def loss(x_, g_):
        y = nb.grid_pull(x_, g_, 3, "dct2", False, prefilter=True)
        z = nb.grid_push(y, g_, None, 3, "dct2", False)
        return (z * w).sum()

    xr = x.clone().requires_grad_(True)
    gr = grid.clone().requires_grad_(True)
    loss(xr, gr).backward()
    rng = np.random.default_rng(1)
    eps = 1e-5
    for _ in range(6):
        i = tuple(int(v) for v in rng.integers(0, 24, 3))
        c = int(rng.integers(0, 3))
        xp, xm = x.clone(), x.clone()
        xp[(0, c) + i] += eps
        xm[(0, c) + i] -= eps
        fd = (loss(xp, grid) - loss(xm, grid)).item() / (2 * eps)
        an = xr.grad[(0, c) + i].item()
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (fd, an)
        d = int(rng.integers(0, 3))
        gp, gm = grid.clone(), grid.clone()
        gp[(0,) + i + (d,)] += eps
        gm[(0,) + i + (d,)] -= eps
        fd = (loss(x, gp) - loss(x, gm)).item() / (2 * eps)
        an = gr.grad[(0,) + i + (d,)].item()
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(fd)), (fd, an)
