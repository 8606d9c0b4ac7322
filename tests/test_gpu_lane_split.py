"""Pull-backward kernels with the last axis' taps spread over lanes, against
the FP64 oracle, at the channel counts and flags that select them:

  * linear, 3-D, 1-4 channels: scalar reductions, two lanes per point (5
    channels take the thread-per-point kernel);
  * cubic, 3-D, 2-4 channels, float32 with a workspace: vector reductions
    into the channel-interleaved accumulator, four lanes per point;
  * linear self-composition backward of velocity exponentiation (covered by
    the SVF tests) shares the first form.

Batches of two, both gradients and each alone, with and without
extrapolation, sorted and natural processing orders.  Tolerance: float32
1e-5 relative (max |err| / max |ref|)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from nitorch_b200 import spatial
from tests._cases import make_case
from tests._gpu_ops import cu, enums, np64, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("C", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("bound", [2, 7, 5])
@pytest.mark.parametrize("ex", [0, 1])
def test_lane_split_pull_backward_vs_oracle(order, C, bound, ex):
    vol, grid = make_case(3, seed=900 + 10 * C + bound + order, in_size=11, out_size=9, C=C, N=2)
    g = np.random.default_rng(C + order)
    grad = g.standard_normal((2, C) + grid.shape[1:-1])
    ref_in, ref_grid = O.grid_pull_backward(grad, vol, grid, [bound], [order], ex)
    b, o = enums(bound, order)
    for mode in ("natural", "sorted"):
        prev = spatial._sample_order_mode
        spatial.set_sample_order(mode)
        try:
            for need_in, need_grid in ((True, True), (True, False), (False, True)):
                V = cu(vol, torch.float32, need_in)
                G = cu(grid, torch.float32, need_grid, grid=True)
                out = spatial.grid_pull_backward(cu(grad, torch.float32), V, G, b, o, ex)
                k = 0
                if need_in:
                    assert relerr(np64(out[k]), ref_in) < 1e-5, (mode, "input")
                    k += 1
                if need_grid:
                    assert relerr(np64(out[k]), ref_grid) < 1e-5, (mode, "grid")
        finally:
            spatial.set_sample_order(prev)


@pytest.mark.parametrize("C", [2, 3, 4])
@pytest.mark.parametrize("mode", ["natural", "sorted"])
def test_lane_split_pull_backward_bf16_vs_oracle(C, mode):
    """bfloat16 cubic images of 2-4 channels (the vector-reduction lane-split
    kernel in natural order, the brick kernels in sorted order) against the
    oracle on the stored (rounded) inputs: the bfloat16 image gradient within
    2^-8 + 1e-5, the float32 grid gradient within 1e-5."""
    vol, grid = make_case(3, seed=950 + C, in_size=11, out_size=9, C=C, N=2)
    grad = np.random.default_rng(C).standard_normal((2, C) + grid.shape[1:-1])
    V = cu(vol, torch.bfloat16, True)
    T = cu(grad, torch.bfloat16)
    G = cu(grid, torch.float32, True, grid=True)
    ref_in, ref_grid = O.grid_pull_backward(np64(T), np64(V), grid.astype(np.float32).astype(np.float64),
                                            [2], [3], 1)
    b, o = enums(2, 3)
    prev = spatial._sample_order_mode
    spatial.set_sample_order(mode)
    try:
        gi, gg = spatial.grid_pull_backward(T, V, G, b, o, 1)
    finally:
        spatial.set_sample_order(prev)
    assert gi.dtype == torch.bfloat16
    assert relerr(np64(gi), ref_in) < 2.0 ** -8 + 1e-5
    assert relerr(np64(gg), ref_grid) < 1e-5
