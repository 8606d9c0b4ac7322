"""The 64-bit offset kernel instances (runtime order, int64 index arithmetic)
against the FP64 oracle.

A call takes them when the grid has 2^31 points or more, or when a tensor's
largest element offset does not fit in 32 bits.  Here the image's second
batch item starts at element 2^31 of one 8 GiB buffer, so every op on it
runs the 64-bit instances; the grid and the other tensors are small.

Tolerances: float32 1e-5 relative (max |err| / max |ref|); order 0
bit-exact against the oracle's float32 build."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from nitorch_b200 import _lib, spatial
from tests._cases import make_case
from tests._gpu_ops import cu, enums, np64, relerr

pytestmark = pytest.mark.gpu

SHAPE = (6, 7, 8)
C = 2


@pytest.fixture(scope="module")
def wide_buffer():
    buf = torch.zeros(2 ** 31 + 4096, dtype=torch.float32, device="cuda")
    yield buf
    del buf
    torch.cuda.empty_cache()


def _wide_image(buf, vol):
    """(2, C, *SHAPE) view whose item 1 starts at element 2^31 of `buf`."""
    n = int(np.prod(SHAPE))
    v = buf.as_strided((2, C) + SHAPE, (2 ** 31, n, SHAPE[1] * SHAPE[2], SHAPE[2], 1))
    v.copy_(torch.as_tensor(vol, dtype=torch.float32))
    return v


@pytest.mark.parametrize("order", [0, 1, 3])
@pytest.mark.parametrize("bound", [2, 7, 5])
def test_wide_offsets_vs_oracle(wide_buffer, order, bound):
    _, grid = make_case(3, seed=700 + 10 * bound + order, in_size=7, out_size=5, C=C, N=2)
    vol = np.random.default_rng(order).standard_normal((2, C) + SHAPE)
    V = _wide_image(wide_buffer, vol)
    b, o = enums(bound, order)
    G = cu(grid, torch.float32)
    out = spatial.grid_pull(V, G, b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    ref = O.grid_pull(vol, grid, [bound], [order], 1)
    assert relerr(np64(out), ref) < 1e-5
    if order == 0:
        ref32 = O.grid_pull(vol.astype(np.float32), grid.astype(np.float32), [bound], [order], 1, real="f32")
        assert np.array_equal(out.cpu().numpy(), ref32)
    # push from a wide input, and the pull's backward pass with a wide image
    tgt = np.random.default_rng(order + 1).standard_normal((2, C) + grid.shape[1:-1])
    T = cu(tgt, torch.float32)
    Vt = V.detach()
    Vt.requires_grad_(True)
    Gr = cu(grid, torch.float32, True)
    dx, dg = spatial.grid_pull_backward(T, Vt, Gr, b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    ref_in, ref_grid = O.grid_pull_backward(tgt, vol, grid, [bound], [order], 1)
    assert relerr(np64(dx), ref_in) < 1e-5
    assert relerr(np64(dg), ref_grid) < 1e-5
    # the same image as the push input (wide target values)
    tv = wide_buffer.as_strided((2, C) + grid.shape[1:-1], (2 ** 31, int(np.prod(grid.shape[1:-1])),
                                                            grid.shape[2] * grid.shape[3], grid.shape[3], 1))
    tv.copy_(torch.as_tensor(tgt, dtype=torch.float32))
    pushed = spatial.grid_push(tv, G, list(SHAPE), b, o, 1)
    assert "order=-1" in _lib.last_kernel(), _lib.last_kernel()
    assert relerr(np64(pushed), O.grid_push(tgt, grid, SHAPE, [bound], [order], 1)) < 1e-5
