"""The fused normal operator pull_push = push(pull(x, grid), grid) and its
backward against the two-call chain grid_pull -> grid_push of the same
library (which the parity suite pins to the oracle), forward and autograd.
Tolerances: float64 1e-11 relative, float32 1e-5 (atomic order); 16-bit
storage 2^-7 (one rounding of the pulled values, as in the chain)."""
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200 as nb
from nitorch_b200 import spatial

pytestmark = pytest.mark.gpu

BOUNDS = ["replicate", "dct1", "dct2", "dst1", "dst2", "dft", "zero"]


def _data(dim, C, ishape, oshape, dtype, seed, jitter=1.3):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((2, C) + ishape, generator=g, dtype=torch.float64)
    scale = torch.tensor([i / o for i, o in zip(ishape, oshape)], dtype=torch.float64)
    grid = nb.identity_grid(oshape, dtype=torch.float64)[None] * scale
    grid = grid.expand(2, *grid.shape[1:]) + jitter * torch.randn((2,) + oshape + (dim,), generator=g,
                                                                   dtype=torch.float64)
    w = torch.randn((2, C) + ishape, generator=g, dtype=torch.float64)
    gdt = torch.float32 if dtype in (torch.bfloat16, torch.float16) else dtype
    return x.to(dtype).cuda(), grid.to(gdt).cuda(), w.to(dtype).cuda()


def _rel(a, b):
    a, b = a.double(), b.double()
    return (a - b).abs().max().item() / max(b.abs().max().item(), 1e-30)


def _both(x, grid, w, order, bound, ex):
    """(z, dx, dgrid) of the fused op and of the chain, loss <z, w>."""
    res = []
    for fused in (True, False):
        xr = x.detach().clone().requires_grad_(True)
        gr = grid.detach().clone().requires_grad_(True)
        if fused:
            z = nb.pull_push(xr, gr, order, bound, ex)
        else:
            z = nb.grid_push(nb.grid_pull(xr, gr, order, bound, ex), gr, x.shape[2:], order, bound, ex)
        (z.float() * w.float()).sum().backward()
        res.append((z.detach(), xr.grad, gr.grad))
    return res


CASES = [(1, (17,), (23,)), (2, (11, 13), (9, 14)), (3, (9, 10, 8), (8, 11, 7))]


@pytest.mark.parametrize("order", range(8))
@pytest.mark.parametrize("case", CASES, ids=["1d", "2d", "3d"])
def test_fused_equals_chain_f64(order, case):
    dim, ishape, oshape = case
    for bi, bound in enumerate(BOUNDS):
        x, grid, w = _data(dim, 3, ishape, oshape, torch.float64, seed=order * 31 + bi + dim)
        for ex in (False, True):
            (zf, dxf, dgf), (zc, dxc, dgc) = _both(x, grid, w, order, bound, ex)
            assert _rel(zf, zc) < 1e-11, (bound, ex)
            assert _rel(dxf, dxc) < 1e-11, (bound, ex)
            assert _rel(dgf, dgc) < 1e-10, (bound, ex)


@pytest.mark.parametrize("order", [1, 3, 5])
def test_fused_equals_chain_f32_mixed_orders(order):
    x, grid, w = _data(3, 4, (20, 18, 16), (20, 18, 16), torch.float32, seed=order)
    o = [order, (order + 1) % 8, 2]
    (zf, dxf, dgf), (zc, dxc, dgc) = _both(x, grid, w, o, ["dct2", "dft", "zero"], True)
    assert _rel(zf, zc) < 1e-5
    assert _rel(dxf, dxc) < 1e-5
    assert _rel(dgf, dgc) < 1e-4


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_fused_equals_chain_16bit(dtype):
    x, grid, w = _data(3, 3, (24, 20, 18), (24, 20, 18), dtype, seed=7)
    (zf, dxf, dgf), (zc, dxc, dgc) = _both(x, grid, w, 3, "dct2", False)
    assert zf.dtype == dtype and dxf.dtype == dtype
    assert _rel(zf, zc) < 2.0 ** -7
    assert _rel(dxf, dxc) < 2.0 ** -7
    assert _rel(dgf, dgc) < 2.0 ** -6


def test_fused_is_self_adjoint():
    x, grid, w = _data(3, 2, (12, 13, 11), (10, 12, 14), torch.float64, seed=5)
    for order in (1, 3):
        a = (nb.pull_push(x, grid, order, "dct2") * w).sum()
        b = (x * nb.pull_push(w, grid, order, "dct2")).sum()
        assert abs((a - b).item()) <= 1e-12 * abs(a.item())


@pytest.mark.parametrize("order", [0, 1, 2, 3])
@pytest.mark.parametrize("bound", ["dct2", "dft", "zero"])
def test_fused_gradcheck(order, bound):
    x, grid, _ = _data(3, 2, (3, 4, 3), (3, 3, 4), torch.float64, seed=order, jitter=1.0)
    x.requires_grad_(True)
    grid.requires_grad_(True)
    # float64 atomics make the scatter order (and the last bits) vary
    assert gradcheck(nb.pull_push, (x, grid, order, bound, True), nondet_tol=1e-12)


def test_fused_deterministic_bit_stable():
    x, grid, w = _data(3, 3, (32, 30, 28), (32, 30, 28), torch.float32, seed=11, jitter=3.0)
    spatial.set_deterministic(True)
    try:
        outs = []
        for _ in range(2):
            xr = x.clone().requires_grad_(True)
            gr = grid.clone().requires_grad_(True)
            z = nb.pull_push(xr, gr, 3, "dct2")
            (z * w).sum().backward()
            outs.append((z, xr.grad, gr.grad))
    finally:
        spatial.set_deterministic(False)
    for a, b in zip(*outs):
        assert torch.equal(a, b)
    zc = nb.grid_push(nb.grid_pull(x, grid, 3, "dct2"), grid, x.shape[2:], 3, "dct2")
    assert _rel(outs[0][0], zc) < 1e-5


def test_fused_sorted_equals_natural():
    x, grid, w = _data(3, 2, (40, 36, 32), (40, 36, 32), torch.float32, seed=13, jitter=4.0)
    b, o = [spatial.BoundType.dct2], [spatial.InterpolationType(3)]
    out = {}
    try:
        for mode in ("natural", "sorted"):
            spatial.set_sample_order(mode)
            out[mode] = spatial.grid_pull_push(x, grid, b, o, 0)
    finally:
        spatial.set_sample_order("auto")
    assert _rel(out["sorted"], out["natural"]) < 1e-5
