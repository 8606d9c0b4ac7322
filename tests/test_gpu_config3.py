"""Full-size affine workload (2-D 4x8x512^2 and 3-D 2x1x128^3, random
affine grids about the field-of-view centre with the shift scaled towards
10 % of the samples outside): every order 0-7 and bound.

pull is checked point by point against the oracle on 512 random sampling
points per batch item (a pulled value depends only on its own point, so the
subset check is exact at full size): float32 within 1e-5 relative to the
float64 oracle on the same stored inputs, order 0 bit-exact against the
oracle's float32 build.  push and count are checked at full size through
their adjoint identities <pull x, y> = <x, push y> and
<count, x> = <1, pull x> (float64 sums of the float32 outputs, 1e-5)."""
import numpy as np
import pytest
import torch

from nitorch_b200 import spatial, workloads
from nitorch_b200.enums import BoundType, InterpolationType
from oracle import oracle as O
from tests._cases import BOUNDS

pytestmark = pytest.mark.gpu

_DATA = {}


def _config3(dim):
    if dim not in _DATA:
        x, grid = workloads.config3(dim)
        xs, gs = x.float(), grid.float()
        g = torch.Generator().manual_seed(23)
        pts = [torch.randint(0, s, (x.shape[0], 512), generator=g) for s in grid.shape[1:-1]]
        y = torch.rand((x.shape[0], x.shape[1], *grid.shape[1:-1]), generator=torch.Generator().manual_seed(24))
        _DATA[dim] = (xs.cuda(), gs.cuda(), y.float().cuda(), pts, xs.double().numpy(), gs.double().numpy())
    return _DATA[dim]


def _subset_grid(gnp, pts):
    """(N, n, 1[, 1], D) grid of the selected sampling points."""
    idx = (np.arange(gnp.shape[0])[:, None],) + tuple(p.numpy() for p in pts)
    sub = gnp[idx]
    return sub[:, :, None, :] if gnp.shape[-1] == 2 else sub[:, :, None, None, :]


def _subset_out(out, pts):
    """(N, C, n) values of a pulled image at the selected points."""
    o = out.cpu()
    vals = [o[n][(slice(None),) + tuple(p[n] for p in pts)] for n in range(o.shape[0])]
    return torch.stack(vals).double().numpy()


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", range(8))
def test_config3_pull_pointwise(dim, order):
    x, grid, _, pts, xnp, gnp = _config3(dim)
    gsub = _subset_grid(gnp, pts)
    for name, code in BOUNDS.items():
        b, o = [BoundType(code)], [InterpolationType(order)]
        mine = _subset_out(spatial.grid_pull(x, grid, b, o, 0), pts)
        ref = O.grid_pull(xnp, gsub, [code], [order], 0).reshape(mine.shape)
        err = np.abs(mine - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err < 1e-5, (name, err)
        if order == 0:
            r32 = O.grid_pull(xnp.astype(np.float32), gsub.astype(np.float32), [code], [0], 0,
                              real="f32").reshape(mine.shape).astype(np.float32)
            assert np.array_equal(mine.astype(np.float32).view(np.uint32), r32.view(np.uint32)), name


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", range(8))
def test_config3_push_count_adjoint(dim, order):
    x, grid, y, *_ = _config3(dim)
    shape = list(x.shape[2:])
    for name, code in BOUNDS.items():
        b, o = [BoundType(code)], [InterpolationType(order)]
        px = spatial.grid_pull(x, grid, b, o, 0)
        py = spatial.grid_push(y, grid, shape, b, o, 0)
        a1 = (px.double() * y.double()).sum().item()
        a2 = (x.double() * py.double()).sum().item()
        assert abs(a1 - a2) <= 1e-5 * max(abs(a1), 1e-30), (name, a1, a2)
        cnt = spatial.grid_count(grid, shape, b, o, 0)
        x0 = x[:, :1].contiguous()
        c1 = (cnt.double() * x0.double()).sum().item()
        c2 = spatial.grid_pull(x0, grid, b, o, 0).double().sum().item()
        assert abs(c1 - c2) <= 1e-5 * max(abs(c2), 1e-30), (name, c1, c2)
