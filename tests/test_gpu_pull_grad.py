"""The fused forward pull + grid_grad (pp_grid_pull_grad): both outputs from
one pass over each point's taps.

Against the separate grid_pull / grid_grad calls on the same inputs (the same
fused multiply-add chains: 1e-6 relative), the FP64 oracle (float64 images:
1e-10; float32: 1e-5), 1/2/3-D, orders 0-7, several bounds, with and
without extrapolation; autograd against the sum of the two separate backward
passes; bfloat16 storage."""
import numpy as np
import pytest
import torch

import nitorch_b200 as nb
from nitorch_b200 import spatial
from oracle import oracle as O
from tests._gpu_ops import cu, enums, np64, relerr

pytestmark = pytest.mark.gpu


def _case(seed, dim, C=2, src=(7, 6, 5), out=(5, 4, 6)):
    r = np.random.default_rng(seed)
    src, out = src[:dim], out[:dim]
    vol = r.standard_normal((2, C) + src)
    grid = -1.5 + r.random((2,) + out + (dim,)) * (np.array(src, np.float64) + 2.0)
    return vol, grid


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [0, 1, 2, 3, 5, 7])
@pytest.mark.parametrize("bound", [2, 5, 7, 3])
@pytest.mark.parametrize("ex", [0, 1])
def test_pull_grad_vs_separate_and_oracle(dim, order, bound, ex):
    vol, grid = _case(100 * dim + 10 * order + bound, dim)
    b, o = enums(bound, order)
    for dt, tol in ((torch.float64, 1e-10), (torch.float32, 1e-5)):
        V, G = cu(vol, dt), cu(grid, dt, grid=True)
        pulled, grad = spatial.grid_pull_grad(V, G, b, o, ex)
        assert relerr(np64(pulled), np64(spatial.grid_pull(V, G, b, o, ex))) < 1e-6
        assert relerr(np64(grad), np64(spatial.grid_grad(V, G, b, o, ex))) < 1e-6
        assert relerr(np64(pulled), O.grid_pull(vol, grid, [bound], [order], ex)) < tol
        assert relerr(np64(grad), O.grid_grad(vol, grid, [bound], [order], ex)) < tol


@pytest.mark.parametrize("order", [1, 3])
def test_pull_grad_autograd(order):
    vol, grid = _case(7 + order, 3)
    x = cu(vol, torch.float64, True)
    g = cu(grid, torch.float64, True, grid=True)
    p, d = nb.grid_pull_grad(x, g, order, "dct2", True)
    wp = torch.randn(p.shape, dtype=torch.float64, device="cuda")
    wd = torch.randn(d.shape, dtype=torch.float64, device="cuda")
    gx, gg = torch.autograd.grad((p * wp).sum() + (d * wd).sum(), (x, g))
    x2 = x.detach().requires_grad_(True)
    g2 = g.detach().requires_grad_(True)
    p2 = nb.grid_pull(x2, g2, order, "dct2", True)
    d2 = nb.grid_grad(x2, g2, order, "dct2", True)
    gx2, gg2 = torch.autograd.grad((p2 * wp).sum() + (d2 * wd).sum(), (x2, g2))
    assert relerr(np64(gx), np64(gx2)) < 1e-10
    assert relerr(np64(gg), np64(gg2)) < 1e-10


def test_pull_grad_bf16_and_api_broadcast():
    vol, grid = _case(5, 3, C=3)
    vb = torch.as_tensor(vol).bfloat16()
    p, d = nb.grid_pull_grad(vb.cuda(), cu(grid, torch.float32, grid=True), 3, "dct2", False)
    assert p.dtype == torch.bfloat16 and d.dtype == torch.bfloat16
    vr = vb.double().numpy()
    assert relerr(np64(p), O.grid_pull(vr, grid, [2], [3], 0)) < 2.0 ** -8
    assert relerr(np64(d), O.grid_grad(vr, grid, [2], [3], 0)) < 2.0 ** -8
    # the public API's broadcasting and prefilter, as grid_pull / grid_grad
    x = torch.randn((3, 9, 8, 7), device="cuda")
    gr = torch.rand((2, 4, 5, 6, 3), device="cuda") * 6
    p, d = nb.grid_pull_grad(x, gr, 3, "dct2", False, prefilter=True)
    assert relerr(np64(p), np64(nb.grid_pull(x, gr, 3, "dct2", False, prefilter=True))) < 1e-6
    assert relerr(np64(d), np64(nb.grid_grad(x, gr, 3, "dct2", False, prefilter=True))) < 1e-6
