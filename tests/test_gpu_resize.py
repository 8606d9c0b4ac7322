"""Separable resize kernel (pp_resize: diagonal affine map, three 1-D passes
over TMA-staged tiles) against the per-point affine pull on the same map
and against the FP64 oracle.

The two CUDA paths evaluate the same fused multiply-add chains (x innermost,
then y, then z, weights from the same stencil), so they agree to float32
rounding (1e-6 relative here; in practice bit for bit).  Cases cover orders
0-3, five bounds, with and without extrapolation, up- and down-sampling
and non-integer steps, batches and channels, z extents that allow TMA
copies (a multiple of 4) and ones that do not, channel-last inputs and
bfloat16 storage.  Tolerance against the oracle: float32 1e-5 relative."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
import nitorch_b200 as nb
from nitorch_b200 import _lib, affine
from nitorch_b200.enums import BoundType
from tests._gpu_ops import np64, relerr

pytestmark = pytest.mark.gpu


def _diag(scales, shifts):
    mat = torch.zeros((1, 3, 4), dtype=torch.float32)
    for d in range(3):
        mat[0, d, d] = scales[d]
        mat[0, d, 3] = shifts[d]
    return mat.cuda()


MAPS = {
    "up2": ((0.5, 0.5, 0.5), (-0.25, -0.25, -0.25), 2.0),
    "down2": ((2.0, 2.0, 2.0), (0.5, 0.5, 0.5), 0.5),
    "odd": ((0.8, 1.3, 0.7), (0.3, -1.2, 0.45), None),
}


def _shape(inshape, m):
    scales, _, f = MAPS[m]
    if f is not None:
        return tuple(max(1, int(s * f)) for s in inshape)
    return tuple(max(1, int(s / sc)) for s, sc in zip(inshape, scales))


@pytest.mark.parametrize("order", [0, 1, 2, 3])
@pytest.mark.parametrize("bound", [2, 7, 5, 0, 3])
@pytest.mark.parametrize("ex", [0, 1])
@pytest.mark.parametrize("m", ["up2", "down2", "odd"])
@pytest.mark.parametrize("zlen", [40, 37])
def test_resize_equals_affine_pull(order, bound, ex, m, zlen):
    g = torch.Generator().manual_seed(order + 10 * bound + zlen)
    inshape = (19, 26, zlen)
    x = torch.randn((2, 3, *inshape), generator=g).cuda()
    scales, shifts, _ = MAPS[m]
    shape = _shape(inshape, m)
    bnd = BoundType(bound)
    out = affine.resize_pull(x, scales, shifts, shape, order, bnd, ex)
    kern = _lib.last_kernel()
    assert kern.startswith("resize_sep_kernel"), kern
    if zlen % 4 == 0:
        assert "tma" in kern, kern
    ref = affine.affine_pull(x, _diag(scales, shifts), shape, order, bnd, ex)
    assert relerr(np64(out), np64(ref)) < 1e-6
    assert affine.resize_status() == 0


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("bound", [2, 5])
def test_resize_vs_oracle(order, bound):
    g = torch.Generator().manual_seed(100 + order + bound)
    inshape = (11, 13, 16)
    x = torch.randn((1, 2, *inshape), generator=g, dtype=torch.float64)
    scales, shifts, _ = MAPS["odd"]
    shape = _shape(inshape, "odd")
    out = affine.resize_pull(x.float().cuda(), scales, shifts, shape, order, BoundType(bound), 0)
    mesh = np.stack(np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij"), -1)
    sc = np.array(scales, np.float32).astype(np.float64)
    sh = np.array(shifts, np.float32).astype(np.float64)
    grid = (mesh * sc + sh)[None]
    ref = O.grid_pull(x.numpy(), grid, [bound], [order], 0)
    assert relerr(np64(out), ref) < 1e-5


def test_resize_channel_last_and_bf16():
    g = torch.Generator().manual_seed(7)
    x = torch.randn((1, 20, 24, 32, 3), generator=g).cuda().movedim(-1, 1)  # channel-last: no TMA
    scales, shifts, _ = MAPS["up2"]
    shape = _shape(x.shape[2:], "up2")
    out = affine.resize_pull(x, scales, shifts, shape, 3, "dct2", 0)
    assert "tma" not in _lib.last_kernel()
    ref = affine.affine_pull(x, _diag(scales, shifts), shape, 3, "dct2", 0)
    assert relerr(np64(out), np64(ref)) < 1e-6
    xb = x.contiguous().bfloat16()
    outb = affine.resize_pull(xb, scales, shifts, shape, 3, "dct2", 0)
    refb = affine.affine_pull(xb, _diag(scales, shifts), shape, 3, "dct2", 0)
    assert relerr(np64(outb), np64(refb)) < 2.0 ** -8


def test_resize_api_and_gradient():
    """nitorch's resize signature routes 3-D float images to the separable
    kernel; its image gradient is the affine push."""
    g = torch.Generator().manual_seed(9)
    x = torch.randn((1, 2, 17, 20, 24), generator=g).cuda().requires_grad_(True)
    y = nb.resize(x, factor=1.5, anchor="c", interpolation=3, bound="dct2", prefilter=False)
    assert _lib.last_kernel().startswith("resize_sep_kernel")
    w = torch.randn(y.shape, generator=g).cuda()
    (y * w).sum().backward()
    dx_sep = x.grad.clone()
    # the same map through the generic affine path
    _, _, scales, shifts = nb.api._resize_transform(list(x.shape[2:]), 1.5, None, "c")
    x2 = x.detach().clone().requires_grad_(True)
    y2 = affine.affine_pull(x2, _diag(scales, shifts), y.shape[2:], 3, "dct2", False)
    assert relerr(np64(y), np64(y2)) < 1e-6
    (y2 * w).sum().backward()
    assert relerr(np64(dx_sep), np64(x2.grad)) < 1e-6
