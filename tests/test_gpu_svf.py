"""Scaling-and-squaring exponentiation of stationary velocity fields
(nitorch.spatial.exp) on the CUDA self-composition kernels against the
oracle's restatement (FP64), plus gradcheck, inverse consistency and
central finite differences of a config-5 style objective (velocity ->
exp -> pull of a moving image at order 3 -> MSE) on a 32^3 crop.
Tolerances: float64 1e-10 relative, float32 1e-5 (one composition) /
1e-4 (eight chained compositions)."""
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200 as nb
from nitorch_b200 import svf, workloads
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

BOUNDS = {"dft": 5, "dct2": 2, "replicate": 0, "zero": 7}


def _vel(shape, seed, scale=2.0, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    D = len(shape)
    v = torch.randn((1, *shape, D), generator=g, dtype=torch.float64)
    if D == 3:
        v = torch.nn.functional.avg_pool3d(v.movedim(-1, 1), 3, 1, 1).movedim(1, -1)
    return (scale * v).to(dtype).cuda()


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bound", list(BOUNDS))
@pytest.mark.parametrize("order", [1, 3])
def test_compose_and_backward_vs_oracle(dim, bound, order):
    shape = (9, 10, 8)[:dim]
    u = _vel(shape, seed=dim * 7 + order, scale=1.5)
    g = _vel(shape, seed=99, scale=1.0)
    for ex in (True, False):
        out = svf.compose(u, order, bound, ex).double().cpu().numpy()
        ref = O.svf_compose(u.cpu().numpy(), BOUNDS[bound], order, int(ex))
        assert relerr(out, ref) < 1e-11, ex
        gd = svf.compose_backward(g, u, order, bound, ex).double().cpu().numpy()
        gref = O.svf_compose_backward(g.cpu().numpy(), u.cpu().numpy(), BOUNDS[bound], order, int(ex))
        assert relerr(gd, gref) < 1e-10, ex


def test_compose_float32_and_channel_strides():
    u = _vel((20, 18, 16), seed=3, scale=2.0)
    ref = O.svf_compose(u.cpu().numpy(), 5, 1, 1)
    u32 = u.float()
    assert relerr(svf.compose(u32).double().cpu().numpy(), ref) < 1e-5
    # components stored first (a movedim view): any strides
    uc = u32.movedim(-1, 1).contiguous().movedim(1, -1)
    assert relerr(svf.compose(uc).double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("bound", list(BOUNDS))
def test_compose_float32_linear_kernel(bound):
    """3-D linear float32 self-composition on its dedicated kernel
    (svf_compose_lin3): every bound, with and without extrapolation, on a
    field large enough to leave the volume, and a components-first view."""
    from nitorch_b200 import _lib
    u = _vel((23, 21, 19), seed=31, scale=3.0)
    for ex in (True, False):
        ref = O.svf_compose(u.cpu().numpy(), BOUNDS[bound], 1, int(ex))
        out = svf.compose(u.float(), 1, bound, ex)
        assert _lib.last_kernel().startswith("svf_compose_lin3")
        assert relerr(out.double().cpu().numpy(), ref) < 1e-5, ex
        uc = u.float().movedim(-1, 1).contiguous().movedim(1, -1)
        assert relerr(svf.compose(uc, 1, bound, ex).double().cpu().numpy(), ref) < 1e-5, ex
        # the backward: the push with neighbouring lanes' corners merged
        g = _vel((23, 21, 19), seed=32, scale=1.0)
        gref = O.svf_compose_backward(g.cpu().numpy(), u.cpu().numpy(), BOUNDS[bound], 1, int(ex))
        gd = svf.compose_backward(g.float(), u.float(), 1, bound, ex)
        assert _lib.last_kernel().startswith("svf_compose_backward_lin3")
        assert relerr(gd.double().cpu().numpy(), gref) < 1e-5, ex
        gd = svf.compose_backward(g.float(), uc, 1, bound, ex)
        assert relerr(gd.double().cpu().numpy(), gref) < 1e-5, ex
        # a field held as the first three slots of a four-slot buffer (16-byte loads)
        up = svf._field_like(u.float()).copy_(u.float())
        assert up.stride()[-2] == 4
        assert relerr(svf.compose(up, 1, bound, ex).double().cpu().numpy(), ref) < 1e-5, ex
        gd = svf.compose_backward(g.float(), up, 1, bound, ex)
        assert relerr(gd.double().cpu().numpy(), gref) < 1e-5, ex


def test_compose_linear_kernels_batch_of_two():
    """Two batch items in one call (the backward's corner merge never crosses
    an item: a warp holds the last voxels of item 0 and the first of item 1
    when Z does not divide 32), with a gradient given as a strided view."""
    from nitorch_b200 import _lib
    shape = (13, 11, 7)
    u = torch.cat([_vel(shape, seed=41, scale=2.5), _vel(shape, seed=42, scale=2.5)])
    g = torch.cat([_vel(shape, seed=43, scale=1.0), _vel(shape, seed=44, scale=1.0)])
    gs = g.float().movedim(-1, 1).contiguous().movedim(1, -1)
    for ex in (True, False):
        out = svf.compose(u.float(), 1, "dft", ex)
        gd = svf.compose_backward(gs, u.float(), 1, "dft", ex)
        assert _lib.last_kernel().startswith("svf_compose_backward_lin3")
        for n in range(2):
            un, gn = u[n:n + 1].cpu().numpy(), g[n:n + 1].cpu().numpy()
            assert relerr(out[n:n + 1].double().cpu().numpy(), O.svf_compose(un, 5, 1, int(ex))) < 1e-5
            assert relerr(gd[n:n + 1].double().cpu().numpy(), O.svf_compose_backward(gn, un, 5, 1, int(ex))) < 1e-5


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("bound", ["dft", "dct2"])
def test_compose_backward_float32_paths(order, bound):
    """float32 3-D fields: the vector-reduction path (workspace given, field
    contiguous or components first) and the per-component path (no
    workspace) against the FP64 oracle."""
    import ctypes
    from nitorch_b200 import _lib
    L = _lib.load()
    u = _vel((21, 19, 17), seed=11 + order, scale=2.0)
    g = _vel((21, 19, 17), seed=12, scale=1.0)
    for ex in (True, False):
        gref = O.svf_compose_backward(g.cpu().numpy(), u.cpu().numpy(), BOUNDS[bound], order, int(ex))
        u32, g32 = u.float(), g.float()
        assert relerr(svf.compose_backward(g32, u32, order, bound, ex).double().cpu().numpy(), gref) < 1e-5
        opt = svf._options(order, bound, ex)
        du, dg = _lib.desc(u32), _lib.desc(g32)
        nws = L.pp_svf_workspace_bytes(ctypes.byref(du), 0)
        assert nws >= u32.numel() // 3 * 16
        ws = torch.empty(nws, dtype=torch.uint8, device="cuda")
        outs = {
            "strided": torch.full((1, 3, 21, 19, 17), 7.0, device="cuda").movedim(1, -1),
            "plain": torch.full_like(u32, 7.0),
        }
        for name, out in outs.items():
            for w, n in ((ctypes.c_void_p(ws.data_ptr()), nws), (None, 0)):
                _lib.check(L.pp_svf_compose_backward(ctypes.byref(dg), ctypes.byref(du),
                                                     ctypes.byref(_lib.desc(out)), ctypes.byref(opt),
                                                     _lib.stream_of(u32), w, n))
                assert relerr(out.double().cpu().numpy(), gref) < 1e-5, (name, n, ex)


@pytest.mark.parametrize("inverse", [False, True])
def test_exp_vs_oracle(inverse):
    v = _vel((12, 11, 10), seed=5, scale=3.0)
    out = svf.exp(v, inverse=inverse).double().cpu().numpy()
    ref = O.svf_exp(v.cpu().numpy(), inverse=inverse)
    assert relerr(out, ref) < 1e-10
    out32 = svf.exp(v.float(), inverse=inverse).double().cpu().numpy()
    assert relerr(out32, ref) < 1e-4
    d = svf.exp(v, inverse=inverse, displacement=True).double().cpu().numpy()
    assert relerr(d, O.svf_exp(v.cpu().numpy(), inverse=inverse, displacement=True)) < 1e-10


def test_exp_backward_vs_oracle():
    v = _vel((10, 9, 11), seed=6, scale=3.0)
    g = _vel((10, 9, 11), seed=7, scale=1.0)
    vr = v.clone().requires_grad_(True)
    (svf.exp(vr) * g).sum().backward()
    ref = O.svf_exp_backward(v.cpu().numpy(), g.cpu().numpy())
    assert relerr(vr.grad.cpu().numpy(), ref) < 1e-10


def test_exp_gradcheck():
    v = _vel((4, 5, 4), seed=8, scale=1.0).requires_grad_(True)
    # float64 atomics vary the last bits between runs
    assert gradcheck(lambda x: svf.exp(x, steps=3), (v,), nondet_tol=1e-12)


def test_exp_inverse_composes_to_identity():
    """exp(-v) inverts exp(v) for a smooth field: u_fwd + u_inv o (id + u_fwd)
    ~ 0 in the interior (the oracle gives 0.027 for this field, max
    displacement 1.76 voxels)."""
    g = torch.Generator().manual_seed(9)
    v = workloads.smooth(torch.randn((1, 3, 24, 24, 24), generator=g, dtype=torch.float64), 3.0, 3)
    v = (v / v.abs().max() * 2.0).movedim(1, -1).contiguous().float().cuda()
    fwd = svf.exp(v, displacement=True)
    inv = svf.exp(v, inverse=True, displacement=True)
    comp = fwd + nb.grid_pull(inv.movedim(-1, 1), nb.identity_grid((24,) * 3, device="cuda")[None] + fwd,
                              1, "dft", True).movedim(1, -1)
    assert comp[:, 4:-4, 4:-4, 4:-4].abs().max().item() < 0.03 * 1.76 * 1.2


@pytest.mark.parametrize("order,tol", [(1, 1e-4), (3, 1e-6)])
def test_config5_crop_finite_differences(order, tol):
    """MSE(pull(moving, exp(v)), fixed) on a 32^3 crop, float64: the velocity
    gradient against central differences along a random direction.  The
    velocity is rescaled to a displacement std of ~2 voxels: with the raw
    config-5 field (std 0.03) every sampling point sits next to an integer
    node, where the linear interpolant has a kink and central differences
    across it are meaningless (the oracle shows the same)."""
    v, mov, fix = workloads.config5(shape=(32, 32, 32))
    v = v * (2.0 / v.std())
    v, mov, fix = v.cuda(), mov.cuda(), fix.cuda()

    def loss(vv):
        phi = svf.exp(vv, interpolation=order)
        w = nb.grid_pull(mov, phi, 3, "dct2", False)
        return ((w - fix) ** 2).mean()

    vr = v.clone().requires_grad_(True)
    loss(vr).backward()
    g = torch.Generator().manual_seed(44)
    d = torch.randn(v.shape, generator=g, dtype=torch.float64).cuda()
    eps = 1e-6
    fd = (loss(v + eps * d) - loss(v - eps * d)).item() / (2 * eps)
    an = (vr.grad * d).sum().item()
    assert abs(fd - an) <= tol * max(abs(fd), 1e-12), (fd, an)
