"""Deterministic mode of the batched plans and of the self-composition
backward of velocity exponentiation: int64 fixed-point scatters give
bit-identical results from run to run (eager and CUDA-graph replay).
Against the float-atomic results: float32 1e-5 relative, bfloat16 storage
2^-7; the self-composition against the FP64 oracle: float32 1e-5, float64
1e-10."""
import pytest
import torch

from nitorch_b200 import spatial, svf
from nitorch_b200.batch import PullPushBatch
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

SHAPES = [(12, 14, 10), (9, 16, 11), (15, 8, 13), (10, 10, 10), (7, 12, 9), (16, 11, 8)]
CHANNELS = [1, 2, 3, 4, 2, 5]
ORDERS = [1, 3, 1, 3, 0, 2]
BOUNDS = {"dft": 5, "dct2": 2, "zero": 7}


def _fill(b, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    for i, s in enumerate(b.shapes):
        b.x[i].copy_(torch.randn(b.x[i].shape, generator=g, device="cuda"))
        b.w[i].copy_(torch.randn(b.w[i].shape, generator=g, device="cuda"))
        mesh = torch.stack(torch.meshgrid(*[torch.arange(n, dtype=torch.float32, device="cuda") for n in s],
                                          indexing="ij"), -1)
        b.grid[i].copy_(mesh[None] + 1.2 * torch.randn(b.grid[i].shape, generator=g, device="cuda"))


def _np(t):
    return t.detach().double().cpu().numpy()


def _outs(b):
    return [t.clone() for t in (b.z_flat, b.dx_flat, b.dgrid_flat)]


@pytest.mark.parametrize("form", ["fused", "chain", "percall"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_batch_deterministic_runs_identical(form, dtype):
    ref = PullPushBatch(SHAPES, CHANNELS, ORDERS, dtype=dtype, form=form)
    _fill(ref, seed=5)
    ref.step_eager()
    want = _outs(ref)
    ref.release()
    b = PullPushBatch(SHAPES, CHANNELS, ORDERS, dtype=dtype, form=form, deterministic=True)
    _fill(b, seed=5)
    b.step_eager()
    first = _outs(b)
    b.step_eager()
    for a, t in zip(first, _outs(b)):
        assert torch.equal(a, t)
    f32 = dtype == torch.float32
    for name, a, w in zip(("z", "dx", "dgrid"), first, want):
        assert relerr(_np(a), _np(w)) < (1e-5 if f32 else 2.0 ** -7), name
    # the same from the captured graph
    b.capture()
    for _ in range(2):
        b.step()
    for a, t in zip(first, _outs(b)):
        assert torch.equal(a, t)
    b.release()


def _field(shape, seed, dtype, scale):
    g = torch.Generator().manual_seed(seed)
    D = len(shape)
    v = torch.randn((1, *shape, D), generator=g, dtype=torch.float64)
    if D == 3:
        v = torch.nn.functional.avg_pool3d(v.movedim(-1, 1), 3, 1, 1).movedim(1, -1)
    return (scale * v).to(dtype).cuda()


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_svf_compose_backward_deterministic(dim, order, dtype):
    shape = {1: (300,), 2: (40, 36), 3: (22, 20, 18)}[dim]
    u = _field(shape, seed=dim + 10 * order, dtype=dtype, scale=1.5)
    g = _field(shape, seed=77, dtype=dtype, scale=1.0)
    tol = 1e-10 if dtype == torch.float64 else 1e-5
    for bound in BOUNDS:
        for ex in (True, False):
            ref = O.svf_compose_backward(_np(g), _np(u), BOUNDS[bound], order, int(ex))
            a = svf.compose_backward(g, u, order, bound, ex, deterministic=True)
            b = svf.compose_backward(g, u, order, bound, ex, deterministic=True)
            assert torch.equal(a, b), (bound, ex)
            assert relerr(_np(a), ref) < tol, (bound, ex)
            f = svf.compose_backward(g, u, order, bound, ex, deterministic=False)
            assert relerr(_np(a), _np(f)) < tol, (bound, ex)


def test_svf_compose_backward_deterministic_strided_output():
    """Components-first output and input views go through the same
    fixed-point path (the accumulators keep the field's own order)."""
    import ctypes
    from nitorch_b200 import _lib
    L = _lib.load()
    u = _field((17, 15, 13), seed=3, dtype=torch.float32, scale=2.0)
    g = _field((17, 15, 13), seed=4, dtype=torch.float32, scale=1.0)
    ref = O.svf_compose_backward(_np(g), _np(u), 5, 1, 1)
    gc = g.movedim(-1, 1).contiguous().movedim(1, -1)
    out = torch.full((1, 3, 17, 15, 13), 5.0, device="cuda").movedim(1, -1)
    opt = svf._options(1, "dft", True, _lib.PP_DETERMINISTIC)
    du = _lib.desc(u)
    nws = L.pp_svf_workspace_bytes(ctypes.byref(du), _lib.PP_DETERMINISTIC)
    ws = torch.empty(nws, dtype=torch.uint8, device="cuda")
    _lib.check(L.pp_svf_compose_backward(ctypes.byref(_lib.desc(gc)), ctypes.byref(du), ctypes.byref(_lib.desc(out)),
                                         ctypes.byref(opt), _lib.stream_of(u), ctypes.c_void_p(ws.data_ptr()), nws))
    assert relerr(_np(out), ref) < 1e-5
    # without the workspace: an error, nothing launched
    rc = L.pp_svf_compose_backward(ctypes.byref(_lib.desc(gc)), ctypes.byref(du), ctypes.byref(_lib.desc(out)),
                                   ctypes.byref(opt), _lib.stream_of(u), None, 0)
    assert rc == _lib.PP_ERR_WORKSPACE


def test_exp_backward_deterministic_switch():
    v = _field((20, 18, 16), seed=8, dtype=torch.float32, scale=3.0).requires_grad_(True)
    w = _field((20, 18, 16), seed=9, dtype=torch.float32, scale=1.0)
    grads = []
    spatial.set_deterministic(True)
    try:
        for _ in range(2):
            v.grad = None
            (svf.exp(v) * w).sum().backward()
            grads.append(v.grad.clone())
    finally:
        spatial.set_deterministic(False)
    assert torch.equal(grads[0], grads[1])
    v.grad = None
    (svf.exp(v) * w).sum().backward()
    assert relerr(_np(grads[0]), _np(v.grad)) < 1e-4
