"""Full-size config-2 workload (1x3x192^3 float32, cubic, dct2, prefilter,
grid = identity + smoothed displacement, ~5 % of the points outside), through
the default processing order (brick-major: the brick kernels).

A pulled value, and each grid-gradient entry of the two backward passes,
depends only on its own sampling point (and the whole image), so checking
512 random points against the float64 oracle is exact at full size:
  * the pull of the prefiltered image;
  * the push backward's grid gradient (push of y, incoming gradient dz);
  * the pull backward's grid gradient (pull of c, incoming gradient t).
The oracle prefilters the stored float32 image in float64 (the
line-vectorised restatement pinned to the C oracle).  The push and the pull
backward's image gradient are checked at full size through the adjoint
identity <pull u, v> = <u, push v> (float64 sums of the float32 outputs).
Tolerance: float32 1e-5 relative (max |err| / max |ref|)."""
import numpy as np
import pytest
import torch

from nitorch_b200 import _lib, coeff, spatial, workloads
from nitorch_b200.enums import BoundType, InterpolationType
from oracle import oracle as O
from oracle import prefilter_torch as P
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

B, OR = [BoundType.dct2], [InterpolationType.cubic]
_D = {}


def _data():
    if not _D:
        x, grid = workloads.config2(size=192, channels=3)
        xs, gs = x.float(), grid.float()
        c64 = P.spline_coeff_nd(xs.double(), [3], [3], 3).numpy()
        g = torch.Generator().manual_seed(29)
        pts = [torch.randint(0, 192, (512,), generator=g) for _ in range(3)]
        _D.update(x=xs.cuda(), grid=gs.cuda(), c64=c64, gnp=gs.double().numpy(), pts=pts)
    return _D


def _sub_grid(gnp, pts):
    return gnp[(0,) + tuple(p.numpy() for p in pts)][None, :, None, None, :]  # (1, 512, 1, 1, 3)


def _at(t, pts):
    """(1, C, 512) values of a (1, C, *grid) tensor at the points."""
    return t[0][(slice(None),) + tuple(p.to(t.device) for p in pts)][None].double().cpu().numpy()


def _at_grid(t, pts):
    """(1, 512, 3) grid-gradient entries at the points."""
    return t[0][tuple(p.to(t.device) for p in pts)][None].double().cpu().numpy()


def test_config2_pull_and_grid_gradients_pointwise():
    d = _data()
    c = coeff.spline_coeff_nd(d["x"], [3], [3], dim=3)
    gsub = _sub_grid(d["gnp"], d["pts"])
    y = spatial.grid_pull(c, d["grid"], B, OR, 0)
    assert _lib.last_kernel().startswith("pp_brick_gather_kernel"), _lib.last_kernel()
    ref = O.grid_pull(d["c64"], gsub, [2], [3], 0).reshape(1, 3, 512)
    assert relerr(_at(y, d["pts"]), ref) < 1e-5

    gen = torch.Generator().manual_seed(31)
    dz = torch.randn((1, 3, 192, 192, 192), generator=gen).cuda()
    t = torch.randn((1, 3, 192, 192, 192), generator=gen).cuda()
    yr = y.detach().requires_grad_(True)
    gr = d["grid"].detach().requires_grad_(True)
    _, dg1 = spatial.grid_push_backward(dz, yr, gr, B, OR, 0)
    ysub = _at(y, d["pts"]).reshape(1, 3, 512, 1, 1)
    ref1 = O.grid_push_backward(dz.double().cpu().numpy(), ysub, gsub, [2], [3], 0)[1].reshape(1, 512, 3)
    assert relerr(_at_grid(dg1, d["pts"]), ref1) < 1e-5

    cr = c.detach().requires_grad_(True)
    _, dg2 = spatial.grid_pull_backward(t, cr, gr, B, OR, 0)
    assert _lib.last_kernel().startswith("pp_brick_pullbwd_kernel"), _lib.last_kernel()
    tsub = _at(t, d["pts"]).reshape(1, 3, 512, 1, 1)
    ref2 = O.grid_pull_backward(tsub, d["c64"], gsub, [2], [3], 0, need_input=False)[0].reshape(1, 512, 3)
    assert relerr(_at_grid(dg2, d["pts"]), ref2) < 1e-5


def test_config2_push_and_image_gradient_adjoint():
    d = _data()
    gen = torch.Generator().manual_seed(37)
    u = torch.randn((1, 3, 192, 192, 192), generator=gen).cuda()
    v = torch.randn((1, 3, 192, 192, 192), generator=gen).cuda()
    pu = spatial.grid_pull(u, d["grid"], B, OR, 0)
    pv = spatial.grid_push(v, d["grid"], [192] * 3, B, OR, 0)
    assert _lib.last_kernel().startswith("pp_brick_scatter_kernel"), _lib.last_kernel()
    a1 = (pu.double() * v.double()).sum().item()
    a2 = (u.double() * pv.double()).sum().item()
    assert abs(a1 - a2) <= 1e-5 * abs(a1)
    # the pull backward's image gradient is the push of the incoming gradient
    ur = u.detach().requires_grad_(True)
    (dx,) = spatial.grid_pull_backward(v, ur, d["grid"], B, OR, 0)
    assert relerr(dx.double().cpu().numpy(), pv.double().cpu().numpy()) < 1e-5
