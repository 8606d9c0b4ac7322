"""Gather-form push (3-D, orders 1 and 3, float32 outputs, sorted sample
order with its cell offsets): output voxels sum the interior points of their
cells, the points near the faces / outside are scattered on top.

Checked against the FP64 oracle and against the scatter-only path of the
same library, over bounds, extrapolation, channel counts beyond one channel
pass, batches, pushes into a volume of another shape, and a collapsed grid
(every point in one cell) that takes many staging passes.  Tolerance:
float32 1e-5 relative (summation order)."""
import contextlib

import numpy as np
import pytest
import torch

import nitorch_b200 as nb
from nitorch_b200 import _lib, spatial
from nitorch_b200.enums import BoundType, InterpolationType
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

BOUNDS = {"replicate": 0, "dct1": 1, "dct2": 2, "dst1": 3, "dst2": 4, "dft": 5, "zero": 7}


@contextlib.contextmanager
def path(gather):
    prev = (spatial._sample_order_mode, spatial._gather_push)
    spatial.set_sample_order("sorted")
    spatial.set_gather_push(gather)
    try:
        yield
    finally:
        spatial.set_sample_order(prev[0])
        spatial.set_gather_push(prev[1])


def push(x, grid, shape, bound, order, ex):
    return spatial.grid_push(x, grid, list(shape), [BoundType(bound)], [InterpolationType(order)], ex)


def data(N, C, gshape, oshape, seed, jitter=1.5):
    r = np.random.default_rng(seed)
    scale = np.array([o / g for g, o in zip(gshape, oshape)])
    idg = np.stack(np.meshgrid(*[np.arange(s, dtype=np.float64) for s in gshape], indexing="ij"), -1)
    grid = idg[None] * scale + jitter * r.standard_normal((N,) + gshape + (3,))
    x = r.standard_normal((N, C) + gshape)
    return x, grid


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("bound", ["dct2", "zero", "dft", "replicate", "dst1"])
@pytest.mark.parametrize("ex", [0, 1])
def test_gather_push_vs_oracle(order, bound, ex):
    x, grid = data(2, 3, (20, 17, 24), (20, 17, 24), seed=order * 10 + BOUNDS[bound] + 100 * ex)
    ref = O.grid_push(x, grid, (20, 17, 24), [BOUNDS[bound]], [order], ex)
    X, G = torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda()
    with path(True):
        y = push(X, G, (20, 17, 24), BOUNDS[bound], order, ex)
    with path(False):
        y0 = push(X, G, (20, 17, 24), BOUNDS[bound], order, ex)
    assert relerr(y.double().cpu().numpy(), ref) < 1e-5
    assert relerr(y.double().cpu().numpy(), y0.double().cpu().numpy()) < 1e-5


@pytest.mark.parametrize("C", [1, 4, 5, 9])
@pytest.mark.parametrize("order", [1, 3])
def test_gather_push_channel_passes(C, order):
    x, grid = data(1, C, (12, 18, 21), (12, 18, 21), seed=C + order)
    ref = O.grid_push(x, grid, (12, 18, 21), [2], [order], 1)
    with path(True):
        y = push(torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda(), (12, 18, 21), 2,
                 order, 1)
    assert relerr(y.double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("oshape", [(30, 9, 40), (8, 8, 8), (5, 33, 17)])
def test_gather_push_other_shape(oshape):
    """Push into a volume of another shape than the grid's (partial CTA
    blocks along every axis)."""
    x, grid = data(2, 2, (14, 13, 12), oshape, seed=sum(oshape), jitter=0.8)
    ref = O.grid_push(x, grid, oshape, [2], [3], 1)
    with path(True):
        y = push(torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda(), oshape, 2, 3, 1)
    assert relerr(y.double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("order", [1, 3])
def test_gather_push_collapsed_grid(order):
    """Every sampling point in one interior cell: one CTA's cells hold all
    points (many staging passes), all other blocks hold none."""
    N, C, gshape, oshape = 1, 2, (24, 20, 16), (12, 12, 12)
    r = np.random.default_rng(order)
    grid = np.empty((N,) + gshape + (3,))
    grid[...] = np.array([5.3, 6.7, 4.2]) + 0.4 * r.random((N,) + gshape + (3,))
    x = r.standard_normal((N, C) + gshape)
    ref = O.grid_push(x, grid, oshape, [2], [order], 0)
    with path(True):
        y = push(torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda(), oshape, 2, order, 0)
    assert relerr(y.double().cpu().numpy(), ref) < 1e-5


def test_gather_push_runs_gather_kernel():
    """With the cell offsets cached, a gather push is two launches (gather,
    residual scatter); the scatter-only push is one."""
    x, grid = data(1, 3, (16, 16, 16), (16, 16, 16), seed=7)
    X, G = torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda()
    L = _lib.load()
    with path(True):
        push(X, G, (16, 16, 16), 2, 3, 1)  # computes and caches the order
        n0 = L.pp_kernel_launches()
        push(X, G, (16, 16, 16), 2, 3, 1)
        n1 = L.pp_kernel_launches()
    with path(False):
        push(X, G, (16, 16, 16), 2, 3, 1)
        n2 = L.pp_kernel_launches()
    assert n1 - n0 == 2
    assert n2 - n1 == 1


def test_gather_push_large_identity_like():
    """A 96^3 grid near the identity, 3 channels: the gather path against
    the scatter path (the oracle is too slow at this size)."""
    g = torch.Generator(device="cuda").manual_seed(3)
    shape = (96, 96, 96)
    grid = nb.identity_grid(shape, dtype=torch.float32, device="cuda")[None]
    grid = grid + 2.0 * torch.randn(grid.shape, generator=g, device="cuda")
    x = torch.randn((1, 3) + shape, generator=g, device="cuda")
    with path(True):
        y = push(x, grid, shape, 2, 3, 1)
    with path(False):
        y0 = push(x, grid, shape, 2, 3, 1)
    assert relerr(y.double().cpu().numpy(), y0.double().cpu().numpy()) < 1e-5


def test_gather_push_autograd_adjoint():
    """<push(x), y> = <x, pull(y)> through the gather path."""
    x, grid = data(1, 3, (18, 22, 19), (18, 22, 19), seed=11, jitter=1.0)
    X, G = torch.from_numpy(x).float().cuda(), torch.from_numpy(grid).float().cuda()
    Y = torch.randn_like(X)
    with path(True):
        px = push(X, G, (18, 22, 19), 2, 3, 1)
        py = spatial.grid_pull(Y, G, [BoundType(2)], [InterpolationType(3)], 1)
    lhs = (px.double() * Y.double()).sum().item()
    rhs = (X.double() * py.double()).sum().item()
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs))
