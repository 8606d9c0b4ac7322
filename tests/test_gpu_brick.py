"""Brick kernels of the cubic 3-D path (push, count and pull backward:
scatter into a shared window; pull, push backward and the pull backward's
grid gradient: gather from a shared window; 1-4 channels) against the FP64
oracle.

The brick kernels run when a 3-D grid comes with the brick-major order
(spatial's "sorted" mode).  Points whose support leaves the brick's window
(near and beyond the volume edges) take the per-point path.  Volumes here
are not multiples of the brick (4 x 4 x 6), grids reach outside the field
of view, batches have two items.  Every call checks that a brick kernel is
the one that ran.

Tolerances: float32 1e-5 relative (max |err| / max |ref|); bfloat16 storage
2^-8 + 1e-5 against the oracle on the rounded inputs."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from nitorch_b200 import _lib, spatial
from tests._cases import identity
from tests._gpu_ops import cu, enums, np64, relerr

pytestmark = pytest.mark.gpu

IN_SHAPE = (21, 22, 27)
OUT_SHAPE = (18, 20, 23)


def _case(seed, C, N=2, spread=1.5, in_shape=IN_SHAPE, out_shape=OUT_SHAPE):
    r = np.random.default_rng(seed)
    vol = r.standard_normal((N, C) + in_shape)
    scale = np.array([(i - 1) / (o - 1) for i, o in zip(in_shape, out_shape)])
    grid = identity(out_shape)[None] * scale + spread * r.standard_normal((N,) + out_shape + (3,))
    return vol, grid


class _Sorted:
    """Brick-major order for every 3-D grid, whatever its size."""

    def __enter__(self):
        self.prev = spatial._sample_order_mode
        spatial.set_sample_order("sorted")
        spatial._orders.clear()

    def __exit__(self, *exc):
        spatial.set_sample_order(self.prev)
        spatial._orders.clear()


def _assert_brick():
    assert _lib.last_kernel().startswith("pp_brick_"), _lib.last_kernel()


@pytest.mark.parametrize("C", [1, 2, 3, 4])
@pytest.mark.parametrize("bound", [2, 7, 5, 3, 0])
@pytest.mark.parametrize("ex", [0, 1])
def test_brick_push_vs_oracle(C, bound, ex):
    vol, grid = _case(1000 + 10 * C + bound, C)
    tgt = np.random.default_rng(C).standard_normal((2, C) + OUT_SHAPE)
    ref = O.grid_push(tgt, grid, IN_SHAPE, [bound], [3], ex)
    b, o = enums(bound, 3)
    with _Sorted():
        out = spatial.grid_push(cu(tgt, torch.float32), cu(grid, torch.float32, grid=True), list(IN_SHAPE),
                                b, o, ex)
        _assert_brick()
    assert relerr(np64(out), ref) < 1e-5


@pytest.mark.parametrize("bound", [2, 7, 5])
@pytest.mark.parametrize("ex", [0, 1])
def test_brick_count_vs_oracle(bound, ex):
    _, grid = _case(1100 + bound, 1)
    ref = O.grid_count(grid, IN_SHAPE, [bound], [3], ex)
    b, o = enums(bound, 3)
    with _Sorted():
        out = spatial.grid_count(cu(grid, torch.float32, grid=True), list(IN_SHAPE), b, o, ex)
        _assert_brick()
    assert relerr(np64(out), ref) < 1e-5


@pytest.mark.parametrize("C", [1, 2, 3, 4])
@pytest.mark.parametrize("bound", [2, 7, 5, 3, 0])
@pytest.mark.parametrize("ex", [0, 1])
def test_brick_pull_backward_vs_oracle(C, bound, ex):
    vol, grid = _case(1200 + 10 * C + bound, C)
    grad = np.random.default_rng(C + 7).standard_normal((2, C) + OUT_SHAPE)
    ref_in, ref_grid = O.grid_pull_backward(grad, vol, grid, [bound], [3], ex)
    b, o = enums(bound, 3)
    with _Sorted():
        for need_in, need_grid in ((True, True), (True, False), (False, True)):
            V = cu(vol, torch.float32, need_in)
            G = cu(grid, torch.float32, need_grid, grid=True)
            out = spatial.grid_pull_backward(cu(grad, torch.float32), V, G, b, o, ex)
            _assert_brick()
            k = 0
            if need_in:
                assert relerr(np64(out[k]), ref_in) < 1e-5, ("input", need_grid)
                k += 1
            if need_grid:
                assert relerr(np64(out[k]), ref_grid) < 1e-5, ("grid", need_in)


@pytest.mark.parametrize("C", [1, 3])
def test_brick_bf16_storage(C):
    """bfloat16 images and gradients (float32 grid): the push and the pull
    backward against the oracle on the bf16-rounded inputs."""
    vol, grid = _case(1300 + C, C)
    r = np.random.default_rng(C)
    grad = r.standard_normal((2, C) + OUT_SHAPE)
    vb = torch.as_tensor(vol).bfloat16().double().numpy()
    gb = torch.as_tensor(grad).bfloat16().double().numpy()
    b, o = enums(2, 3)
    bound = 2.0 ** -8 + 1e-5
    with _Sorted():
        out = spatial.grid_push(cu(gb, torch.bfloat16), cu(grid, torch.float32, grid=True), list(IN_SHAPE), b, o, 1)
        _assert_brick()
        assert relerr(np64(out), O.grid_push(gb, grid, IN_SHAPE, [2], [3], 1)) < bound
        V = cu(vb, torch.bfloat16, True)
        G = cu(grid, torch.float32, True, grid=True)
        din, dgrid = spatial.grid_pull_backward(cu(gb, torch.bfloat16), V, G, b, o, 1)
        _assert_brick()
    ref_in, ref_grid = O.grid_pull_backward(gb, vb, grid, [2], [3], 1)
    assert relerr(np64(din), ref_in) < bound
    assert relerr(np64(dgrid), ref_grid) < 1e-5  # the grid gradient is stored in float32


def test_brick_matches_per_point_path_on_smooth_field():
    """A 64^3 smooth deformation (most points in interior bricks): the brick
    kernel against the per-point kernels (natural order) and the adjoint
    identity <pull x, y> = <x, push y>."""
    from nitorch_b200 import workloads
    x, g = workloads.config2(size=64, channels=3)
    x, g = x.float().cuda(), g.float().cuda()
    y = torch.randn(x.shape, generator=torch.Generator().manual_seed(5)).cuda()
    b, o = enums(2, 3)
    res = {}
    for mode in ("natural", "sorted"):
        prev = spatial._sample_order_mode
        spatial.set_sample_order(mode)
        spatial._orders.clear()
        try:
            push = spatial.grid_push(y, g, list(x.shape[2:]), b, o, 0)
            if mode == "sorted":
                _assert_brick()
            xr = x.detach().requires_grad_(True)
            gr = g.detach().requires_grad_(True)
            din, dgrid = spatial.grid_pull_backward(y, xr, gr, b, o, 0)
            if mode == "sorted":
                _assert_brick()
            pull = spatial.grid_pull(x, g, b, o, 0)
            res[mode] = (push, din, dgrid, pull)
        finally:
            spatial.set_sample_order(prev)
            spatial._orders.clear()
    for a, r in zip(res["sorted"], res["natural"]):
        assert relerr(np64(a), np64(r)) < 1e-5
    push, _, _, pull = res["sorted"]
    lhs = float((pull.double() * y.double()).sum())
    rhs = float((x.double() * push.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(rhs)


@pytest.mark.parametrize("C", [1, 2, 3, 4])
@pytest.mark.parametrize("bound", [2, 7, 5, 3, 0])
@pytest.mark.parametrize("ex", [0, 1])
def test_brick_gathers_vs_oracle(C, bound, ex):
    """Pull through the brick gather kernel; the push backward (per-point
    kernel in brick-major order) on the same inputs."""
    vol, grid = _case(1400 + 10 * C + bound, C)
    r = np.random.default_rng(C + 11)
    y = r.standard_normal((2, C) + OUT_SHAPE)        # pushed values
    dz = r.standard_normal((2, C) + IN_SHAPE)        # gradient of the push output
    b, o = enums(bound, 3)
    ref_pull = O.grid_pull(vol, grid, [bound], [3], ex)
    ref_in, ref_grid = O.grid_push_backward(dz, y, grid, [bound], [3], ex)
    with _Sorted():
        out = spatial.grid_pull(cu(vol, torch.float32), cu(grid, torch.float32, grid=True), b, o, ex)
        _assert_brick()
        assert relerr(np64(out), ref_pull) < 1e-5
        for need_in, need_grid in ((True, True), (True, False), (False, True)):
            Y = cu(y, torch.float32, need_in)
            G = cu(grid, torch.float32, need_grid, grid=True)
            res = spatial.grid_push_backward(cu(dz, torch.float32), Y, G, b, o, ex)
            k = 0
            if need_in:
                assert relerr(np64(res[k]), ref_in) < 1e-5, ("input", need_grid)
                k += 1
            if need_grid:
                assert relerr(np64(res[k]), ref_grid) < 1e-5, ("grid", need_in)


def test_brick_pull_matches_per_point_pull():
    """The brick gather sums the taps in the per-point kernel's order (x,
    then y, then z partial sums, boundary signs folded into the values
    instead of the weights): the two pulls agree to float32 rounding."""
    vol, grid = _case(1500, 3)
    b, o = enums(2, 3)
    V, G = cu(vol, torch.float32), cu(grid, torch.float32, grid=True)
    with _Sorted():
        a = spatial.grid_pull(V, G, b, o, 1)
        _assert_brick()
    prev = spatial._sample_order_mode
    spatial.set_sample_order("natural")
    try:
        r = spatial.grid_pull(V, G, b, o, 1)
    finally:
        spatial.set_sample_order(prev)
    assert relerr(np64(a), np64(r)) < 1e-6
