"""The 64-bit offset kernel instances (runtime order, int64 index arithmetic)
against the FP64 oracle.

Batch offsets are always 64-bit; a call takes the 64-bit instances when the
grid has 2^31 points or more, or when an offset inside one batch item does
not fit in 32 bits.  Here the image is a view of one 8 GiB buffer whose x
axis has a stride of 2^30 elements: its third x plane starts at element
2^31, so every op on it runs the 64-bit instances (checked through
pp_last_kernel); the grid and the other tensors are small.

Tolerances: float32 1e-5 relative (max |err| / max |ref|); order 0
bit-exact against the oracle's float32 build."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from nitorch_b200 import _lib, spatial
from tests._gpu_ops import cu, enums, np64, relerr

pytestmark = pytest.mark.gpu

C = 2
XS = 2 ** 30  # x stride of the wide views (elements)


@pytest.fixture(scope="module")
def wide_buffer():
    buf = torch.zeros(2 * XS + 4096, dtype=torch.float32, device="cuda")
    yield buf
    del buf
    torch.cuda.empty_cache()


def _wide(buf, arr):
    """(1, C, 3, Y, Z) view of `buf` with x stride 2^30, holding `arr`."""
    _, c, x, y, z = arr.shape
    assert x == 3
    v = buf.as_strided(arr.shape, (0, y * z, XS, z, 1))
    v.copy_(torch.as_tensor(arr, dtype=torch.float32))
    return v


def _grid(seed, src, out):
    r = np.random.default_rng(seed)
    lo, hi = -1.0, np.array(src, np.float64)
    return (lo + r.random((1,) + out + (3,)) * (hi + 1.0))


@pytest.mark.parametrize("order", [0, 1, 3])
@pytest.mark.parametrize("bound", [2, 7, 5])
def test_wide_offsets_vs_oracle(wide_buffer, order, bound):
    src = (3, 7, 8)
    out_shape = (3, 6, 5)
    grid = _grid(700 + 10 * bound + order, src, out_shape)
    vol = np.random.default_rng(order).standard_normal((1, C) + src)
    b, o = enums(bound, order)
    G = cu(grid, torch.float32)
    # pull from a wide image
    V = _wide(wide_buffer, vol)
    out = spatial.grid_pull(V, G, b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    assert relerr(np64(out), O.grid_pull(vol, grid, [bound], [order], 1)) < 1e-5
    if order == 0:
        ref32 = O.grid_pull(vol.astype(np.float32), grid.astype(np.float32), [bound], [order], 1, real="f32")
        assert np.array_equal(out.cpu().numpy(), ref32)
    # the pull's backward pass with the wide image
    tgt = np.random.default_rng(order + 1).standard_normal((1, C) + out_shape)
    Vt = V.detach().requires_grad_(True)
    Gr = cu(grid, torch.float32, True)
    dx, dg = spatial.grid_pull_backward(cu(tgt, torch.float32), Vt, Gr, b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    ref_in, ref_grid = O.grid_pull_backward(tgt, vol, grid, [bound], [order], 1)
    assert relerr(np64(dx), ref_in) < 1e-5
    assert relerr(np64(dg), ref_grid) < 1e-5
    # push from a wide input on a 3 x 6 x 5 grid
    T = _wide(wide_buffer, tgt)
    pushed = spatial.grid_push(T, G, list(src), b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    assert relerr(np64(pushed), O.grid_push(tgt, grid, src, [bound], [order], 1)) < 1e-5


@pytest.mark.parametrize("bound", ["dct2", "dft", "zero"])
def test_wide_regularisers_vs_oracle(wide_buffer, bound):
    """The regularisers' 64-bit neighbour-offset instances: a field and a
    displacement grid whose x axis has a stride of 2^30 elements (their ±2
    steps along x do not fit 32 bits)."""
    from nitorch_b200 import solve
    code = {"dct2": 2, "dft": 5, "zero": 7}[bound]
    vol = np.random.default_rng(5).standard_normal((1, C, 3, 7, 8))
    V = _wide(wide_buffer, vol)
    for (a, m, b) in (([0.1], [1.0], [0.0]), ([0.05], [0.3], [0.7])):
        got = solve.c_regulariser(V, None, None, 3, a, m, b, 1.0, [1.2, 0.9, 1.1], bound)
        ref = O.regulariser(vol, None, None, a, m, b, [1.2, 0.9, 1.1], [code])
        assert relerr(got.double().cpu().numpy(), ref) < 1e-5, (a, m, b)
    fld = np.random.default_rng(6).standard_normal((1, 3, 7, 8, 3))
    G = wide_buffer.as_strided(fld.shape, (0, XS, 8 * 3, 3, 1))
    G.copy_(torch.as_tensor(fld, dtype=torch.float32))
    got = solve.c_regulariser_grid(G, None, None, 0.01, 0.2, 0.5, (0.7, 0.4), 1.0, [1.2, 0.9, 1.1], bound)
    ref = O.regulariser_grid(np.moveaxis(fld, -1, 1), None, None, 0.01, 0.2, 0.5, 0.7, 0.4, [1.2, 0.9, 1.1], [code])
    assert relerr(got.double().cpu().numpy(), np.moveaxis(ref, 1, -1)) < 1e-5
