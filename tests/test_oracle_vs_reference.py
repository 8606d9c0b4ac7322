"""Pin the CPU oracle against the reference's own compiled CPU backend.

The reference (nitorch/_C, compiled from its sources by oracle/build_ref.py
into oracle/_ref/) is run on the same seeded float64 inputs as the oracle,
for all eight push/pull functions, 1/2/3-D, seven bounds, orders 0-7.
Reference defects are switched on in the oracle where they apply
(D1: third-axis order, D3: zero second derivatives for orders 5-7), the
D2 workaround (grad with last stride > 1) is used for grid_grad_backward,
and the 1-D out-of-bound stray write (D6) is avoided.
Skipped when the compiled reference is absent (it is never built on a GPU
box; the committed golden fixtures pin the oracle there).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import reference as R
from tests._cases import BOUND_CODES, ORDERS, make_case

ref = R.load_compiled()
pytestmark = pytest.mark.skipif(ref is None, reason="compiled reference not built")

TOL = 1e-11


def _t(a, rg=False):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if rg:
        t.requires_grad_(True)
    return t


def _enums(bound, order):
    B = {v.value: v for v in ref.BoundType.__members__.values()}
    I = {v.value: v for v in ref.InterpolationType.__members__.values()}
    return [B[bound]], [I[order]]


def _close(a, b, tol=TOL):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(1.0, float(np.abs(b).max()) if b.size else 1.0)
    err = float(np.abs(a - b).max()) if a.size else 0.0
    assert err <= tol * scale, f"max abs err {err:.3e} (scale {scale:.3e})"


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bound", BOUND_CODES)
@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("extrapolate", [0, 1])
def test_forward_ops(dim, bound, order, extrapolate):
    vol, grid = make_case(dim, seed=100 * dim + 10 * bound + order)
    b, o = _enums(bound, order)
    # pull
    r = ref.grid_pull(_t(vol), _t(grid), b, o, extrapolate).numpy()
    _close(O.grid_pull(vol, grid, [bound], [order], extrapolate), r)
    # grad (sgrad).  Reference defect D6: in 1-D its out-of-bound branch also
    # zeroes a second gradient component that 1-D outputs do not have
    # (pushpull_common.cpp:1036-1048), i.e. a neighbouring element; skip
    # that combination.
    if not (dim == 1 and extrapolate == 0):
        r = ref.grid_grad(_t(vol), _t(grid), b, o, extrapolate).numpy()
        _close(O.grid_grad(vol, grid, [bound], [order], extrapolate), r)
    # push: input (N,C,*grid)
    tgt = np.random.default_rng(7).standard_normal((1, 2) + grid.shape[1:-1])
    shape = vol.shape[2:]
    r = ref.grid_push(_t(tgt), _t(grid), list(shape), b, o, extrapolate).numpy()
    _close(O.grid_push(tgt, grid, shape, [bound], [order], extrapolate), r)
    # count
    r = ref.grid_count(_t(grid), list(shape), b, o, extrapolate).numpy()
    _close(O.grid_count(grid, shape, [bound], [order], extrapolate), r)


def _last_stride_gt1(a):
    """Copy of `a` laid out (N, C, K, *spatial) in memory, so that the last
    (K) dimension has a stride > 1 -- the workaround for reference defect D2
    (second derivatives only computed when trgt_sK > 1,
    pushpull_common.cpp:1137,1152,1167)."""
    shape = a.shape
    n, c, k = shape[0], shape[1], shape[-1]
    sp = shape[2:-1]
    prod_sp = int(np.prod(sp))
    strides = [c * k * prod_sp, k * prod_sp]
    acc = 1
    sp_strides = []
    for s in reversed(sp):
        sp_strides.insert(0, acc)
        acc *= s
    t = torch.empty_strided(shape, strides + sp_strides + [prod_sp], dtype=torch.float64)
    t.copy_(torch.from_numpy(a))
    assert t.stride(-1) > 1
    return t


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bound", BOUND_CODES)
@pytest.mark.parametrize("order", ORDERS)
def test_backward_ops(dim, bound, order):
    extrapolate = 1
    vol, grid = make_case(dim, seed=1000 + 100 * dim + 10 * bound + order)
    b, o = _enums(bound, order)
    g = np.random.default_rng(9)
    gout = g.standard_normal((1, 2) + grid.shape[1:-1])
    # pull backward
    r = ref.grid_pull_backward(_t(gout), _t(vol, True), _t(grid, True), b, o, extrapolate)
    mine = O.grid_pull_backward(gout, vol, grid, [bound], [order], extrapolate)
    _close(mine[0], r[0].detach().numpy())
    _close(mine[1], r[1].detach().numpy())
    # push backward: grad has the pushed shape (= vol shape)
    tgt = g.standard_normal((1, 2) + grid.shape[1:-1])
    gpush = g.standard_normal(vol.shape)
    r = ref.grid_push_backward(_t(gpush), _t(tgt, True), _t(grid, True), b, o, extrapolate)
    mine = O.grid_push_backward(gpush, tgt, grid, [bound], [order], extrapolate)
    _close(mine[0], r[0].detach().numpy())
    _close(mine[1], r[1].detach().numpy())
    # count backward
    gcount = g.standard_normal((1, 1) + vol.shape[2:])
    r = ref.grid_count_backward(_t(gcount), _t(grid, True), b, o, extrapolate)
    _close(O.grid_count_backward(gcount, grid, [bound], [order], extrapolate), r.detach().numpy())
    # grad backward: D2 workaround (last-dim stride > 1), D3 quirk for orders >= 5
    ggrad = g.standard_normal((1, 2) + grid.shape[1:-1] + (dim,))
    tg = _last_stride_gt1(ggrad)
    r = ref.grid_grad_backward(tg, _t(vol, True), _t(grid, True), b, o, extrapolate)
    mine = O.grid_grad_backward(ggrad, vol, grid, [bound], [order], extrapolate,
                                quirks=O.QUIRK_D3)
    _close(mine[0], r[0].detach().numpy())
    _close(mine[1], r[1].detach().numpy())


@pytest.mark.parametrize("orders", [(1, 1, 3), (3, 2, 1), (0, 3, 5)])
def test_anisotropic_orders_quirk_d1(orders):
    vol, grid = make_case(3, seed=77)
    B = ref.BoundType.dct2
    I = {v.value: v for v in ref.InterpolationType.__members__.values()}
    r = ref.grid_pull(_t(vol), _t(grid), [B], [I[k] for k in orders], 1).numpy()
    _close(O.grid_pull(vol, grid, [2], list(orders), 1, quirks=O.QUIRK_D1), r)


def test_float32_order0_bit_exact():
    """Order 0 and the index maps: float32 oracle == float32 reference, bitwise."""
    for dim in (1, 2, 3):
        for bound in BOUND_CODES:
            vol, grid = make_case(dim, seed=5 + bound, spread=3.0)
            vol32 = vol.astype(np.float32)
            grid32 = grid.astype(np.float32)
            b, o = _enums(bound, 0)
            for ex in (0, 1, 2):
                r = ref.grid_pull(_t(vol32), _t(grid32), b, o, ex).numpy()
                m = O.grid_pull(vol32, grid32, [bound], [0], ex, real="f32")
                assert np.array_equal(m.view(np.uint32), r.view(np.uint32)), (dim, bound, ex)
                tgt = np.random.default_rng(3).standard_normal((1, 2) + grid.shape[1:-1]).astype(np.float32)
                r = ref.grid_push(_t(tgt), _t(grid32), list(vol.shape[2:]), b, o, ex).numpy()
                m = O.grid_push(tgt, grid32, vol.shape[2:], [bound], [0], ex, real="f32")
                # single tap per sample -> atomic order can still reorder sums of
                # several samples landing on one voxel; compare exactly on
                # voxels hit once and to 1 ulp elsewhere
                np.testing.assert_allclose(m, r, rtol=2e-7, atol=1e-7)


def _ref_svf_exp(vel, steps, bound, order):
    """nitorch/spatial/_svf.py:85-94 driven by the reference's own compiled
    grid_pull (the _pull_vel wiring of :323-362: components moved to the
    channel axis, dft bound, extrapolation on)."""
    b, o = [ref.BoundType(bound)], [ref.InterpolationType(order)]
    u = torch.as_tensor(vel) / 2 ** steps
    shape = u.shape[1:-1]
    idg = torch.stack(torch.meshgrid(*[torch.arange(s, dtype=torch.float64) for s in shape], indexing="ij"), -1)
    for _ in range(steps):
        pulled = ref.grid_pull(u.movedim(-1, 1).contiguous(), idg[None] + u, b, o, 1)
        u = u + pulled.movedim(1, -1)
    return (u + idg[None]).numpy()


@pytest.mark.parametrize("bound", [5, 2])
@pytest.mark.parametrize("order", [1, 3])
def test_svf_exp_restatement(bound, order):
    rng = np.random.default_rng(order * 10 + bound)
    vel = rng.standard_normal((1, 7, 8, 6, 3)) * 2.0
    mine = O.svf_exp(vel, steps=6, bound=bound, order=order)
    theirs = _ref_svf_exp(vel, 6, bound, order)
    assert np.abs(mine - theirs).max() / np.abs(theirs).max() < 1e-12


def test_svf_backward_restatement_finite_differences():
    rng = np.random.default_rng(3)
    u = rng.standard_normal((1, 5, 6, 4, 3)) * 0.7
    g, d = rng.standard_normal(u.shape), rng.standard_normal(u.shape)
    an = (O.svf_exp_backward(u, g, steps=3) * d).sum()
    e = 1e-6
    fd = ((O.svf_exp(u + e * d, steps=3) * g).sum() - (O.svf_exp(u - e * d, steps=3) * g).sum()) / (2 * e)
    assert abs(an - fd) <= 1e-8 * abs(fd)
