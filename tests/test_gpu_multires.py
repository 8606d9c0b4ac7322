"""Multigrid resampling on the GPU against the reference's own outputs
(tests/golden/multires_golden.npz) and the float64 oracle.

* fmg_prolongation / fmg_restriction: the separable kernel with the
  multigrid stencils (pp_fmg_*), all seven bounds, 3-D fixtures; 1-D / 2-D
  and a 64 x 80 x 96 volume (interior tiles staged by TMA) against the
  oracle; bfloat16 storage;
* the native resize with its four alignment modes, adjoint and
  normalisation; its prolongation / restriction wrappers and backward;
* the nitorch/_C/resize.py wrappers (factor / shape / displacement-grid
  forms) and the multigrid solvers' prolong / restrict.

Inputs are the fixtures' float64 values stored in float32; tolerance float32
1e-5 relative (max |err| / max |ref|), bfloat16 2^-8."""
import os

import numpy as np
import pytest
import torch

from nitorch_b200 import _lib, multires as M
from nitorch_b200.enums import BoundType, GridAlignType, InterpolationType
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "multires_golden.npz"))
BOUNDS = (0, 1, 2, 3, 4, 5, 7)


def _cu(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a)).to(dtype).cuda()


def _np(t):
    return t.detach().double().cpu().numpy()


@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("b", BOUNDS)
def test_fmg_vs_reference(k, b):
    x = _cu(GOLD[f"fmg_x{k}"])
    p = M.fmg_prolongation(x, None, [BoundType(b)])
    assert _lib.last_kernel().startswith("resize_sep_kernel") and "mode=2" in _lib.last_kernel()
    assert relerr(_np(p), GOLD[f"fmg_pro{k}_b{b}"]) < 1e-5
    r = M.fmg_restriction(x, None, [BoundType(b)])
    assert "mode=1" in _lib.last_kernel()
    assert relerr(_np(r), GOLD[f"fmg_res{k}_b{b}"]) < 1e-5


@pytest.mark.parametrize("shape", [(2, 3, 13), (1, 2, 9, 7), (1, 1, 17, 1)])
@pytest.mark.parametrize("b", (2, 5, 3, 7))
def test_fmg_1d_2d_vs_oracle(shape, b):
    """1-D / 2-D images (the reference raises on them): the operator on the
    real axes, identity on the padded ones."""
    x = np.random.default_rng(len(shape) + b).standard_normal(shape)
    assert relerr(_np(M.fmg_prolongation(_cu(x), None, [BoundType(b)])), O.fmg_prolongation(x, [b])) < 1e-5
    assert relerr(_np(M.fmg_restriction(_cu(x), None, [BoundType(b)])), O.fmg_restriction(x, [b])) < 1e-5


@pytest.mark.parametrize("b", (2, 1, 5))
def test_fmg_volume_vs_oracle(b):
    """1 x 2 x 64 x 80 x 96 float32 (z contiguous, TMA-staged tiles), odd
    target shapes for the restriction, a given output lattice."""
    x = np.random.default_rng(b).standard_normal((1, 2, 64, 80, 96))
    X = _cu(x)
    p = M.fmg_prolongation(X, None, [BoundType(b)])
    assert "tma" in _lib.last_kernel()
    assert relerr(_np(p), O.fmg_prolongation(x, [b])) < 1e-5
    out = torch.empty((1, 2, 33, 41, 47), device="cuda")
    r = M.fmg_restriction(X, out, [BoundType(b)])
    assert r is out
    assert relerr(_np(r), O.fmg_restriction(x, [b], shape=(33, 41, 47))) < 1e-5


def test_fmg_bf16():
    x = np.random.default_rng(7).standard_normal((1, 3, 12, 10, 16))
    xb = torch.as_tensor(x).bfloat16()
    xr = xb.double().numpy()
    p = M.fmg_prolongation(xb.cuda(), None, [BoundType.dct2])
    assert p.dtype == torch.bfloat16
    assert relerr(_np(p), O.fmg_prolongation(xr, [2])) < 2.0 ** -8
    r = M.fmg_restriction(xb.cuda(), None, [BoundType.dct2])
    assert relerr(_np(r), O.fmg_restriction(xr, [2])) < 2.0 ** -8


@pytest.mark.parametrize("mode", range(4))
@pytest.mark.parametrize("adj", (0, 1))
@pytest.mark.parametrize("norm", (0, 1))
@pytest.mark.parametrize("kf", (0, 1))
@pytest.mark.parametrize("order", (1, 3))
def test_native_resize_vs_reference(mode, adj, norm, kf, order):
    fac = (2.0, 0.7)[kf]
    x = _cu(GOLD["rz_x"])
    got = M.resize(x, None, [fac], [BoundType.dct2], [InterpolationType(order)], [GridAlignType(mode)],
                   bool(adj), bool(norm))
    if not adj:
        assert _lib.last_kernel().startswith("resize_sep_kernel"), _lib.last_kernel()
    assert relerr(_np(got), GOLD[f"rz_m{mode}_a{adj}_n{norm}_f{kf}_o{order}"]) < 1e-5


def test_native_wrappers_vs_reference():
    x, xf = _cu(GOLD["rz_x"]), _cu(GOLD["wrap_fine"])
    fine = torch.zeros((1, 2, 10, 12, 14), device="cuda")
    coarse = torch.zeros((1, 2, 5, 6, 7), device="cuda")
    assert relerr(_np(M.prolongation(x, fine.clone())), GOLD["wrap_prolongation"]) < 1e-5
    assert relerr(_np(M.prolongation_backward(xf, coarse.clone())), GOLD["wrap_prolongation_backward"]) < 1e-5
    assert relerr(_np(M.restriction(xf, coarse.clone())), GOLD["wrap_restriction"]) < 1e-5
    assert relerr(_np(M.restriction_backward(x, fine.clone())), GOLD["wrap_restriction_backward"]) < 1e-5
    # resize_backward is resize with the inverse factor and the adjoint flipped
    y = M.resize(x, None, [2.0], [], [], ["edge"], False, False)
    g = torch.randn(y.shape, device="cuda")
    gb = M.resize_backward(g, torch.zeros_like(x), [2.0], [], [], ["edge"], False, False)
    lhs = float((y.double() * g.double()).sum())
    rhs = float((x.double() * gb.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_python_wrappers_vs_reference():
    x, xf = _cu(GOLD["rz_x"]), _cu(GOLD["wrap_fine"])
    assert relerr(_np(M.c_prolongation(x, factor=2., bound="dct1")), GOLD["c_prolongation"]) < 1e-5
    assert relerr(_np(M.c_restriction(xf, factor=2., bound="dft")), GOLD["c_restriction"]) < 1e-5
    assert relerr(_np(M.c_restriction(xf, shape=(4, 7, 5))), GOLD["c_restriction_shape"]) < 1e-5
    v, vf = _cu(GOLD["grid_coarse"]), _cu(GOLD["grid_fine"])
    assert relerr(_np(M.c_prolongation_grid(v)), GOLD["c_prolongation_grid"]) < 1e-5
    assert relerr(_np(M.c_restriction_grid(vf)), GOLD["c_restriction_grid"]) < 1e-5


def test_solver_prolong_restrict_vs_reference():
    import nitorch_b200 as nb
    v, vf = _cu(GOLD["grid_coarse"]), _cu(GOLD["grid_fine"])
    assert relerr(_np(nb.prolong(v, dim=3)), GOLD["sv_prolong"]) < 1e-5
    assert _lib.last_kernel().startswith("resize_sep_kernel"), _lib.last_kernel()
    assert relerr(_np(nb.prolong(v, order=3, bound="dft", dim=3)), GOLD["sv_prolong_o3"]) < 1e-5
    assert relerr(_np(nb.restrict(vf, dim=3)), GOLD["sv_restrict"]) < 1e-5
    assert relerr(_np(nb.restrict(vf, shape=(4, 5, 8), dim=3)), GOLD["sv_restrict_shape"]) < 1e-5
    assert relerr(_np(nb.prolong(v[0])), GOLD["sv_prolong_nobatch"]) < 1e-5
