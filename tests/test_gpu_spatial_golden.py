"""The callers of the push/pull path on the GPU against the reference's own
nitorch.spatial outputs (tests/golden/spatial_golden.npz, generated from the
reference by tests/golden/make_golden.py): grid_jacobian / grid_jacdet by
finite differences (all bounds, both field types, voxel sizes, a singleton
axis) and at sampled coordinates, resize (all anchors, factors, a target
shape, the orientation matrix), reslice, and the velocity exponentiation
with its autograd gradient; plus gradchecks of the Jacobian kernels.
Float64 throughout; tolerance 1e-10 relative (1e-9 for the exponentiation
gradient, eight chained compositions; 1e-6 for the cubic resize against
the reference, whose prefilter carries rounding noise -- the same resize is
checked against the exact FP64 oracle at 1e-11)."""
import os

import numpy as np
import pytest
import torch
from torch.autograd import gradcheck

import nitorch_b200 as nb
from nitorch_b200 import svf
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spatial_golden.npz"))
BOUNDS = ("dft", "dct2", "dct1", "dst1", "dst2", "zero", "replicate")


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("bound", BOUNDS)
@pytest.mark.parametrize("typ", ["grid", "disp"])
def test_jacobian_fd_vs_reference(bound, typ):
    f3, f2 = cu(G["jac_f3"]), cu(G["jac_f2"])
    assert relerr(nb.grid_jacobian(f3, bound=bound, type=typ).cpu().numpy(), G[f"jac3_{bound}_{typ}"]) < 1e-12
    assert relerr(nb.grid_jacdet(f3, bound=bound, type=typ).cpu().numpy(), G[f"jacdet3_{bound}_{typ}"]) < 1e-10
    assert relerr(nb.grid_jacobian(f2, bound=bound, type=typ).cpu().numpy(), G[f"jac2_{bound}_{typ}"]) < 1e-12
    got = nb.grid_jacobian(cu(G["jac_f1s"]), bound=bound, type="disp").cpu().numpy()
    assert relerr(got, G[f"jac1s_{bound}"]) < 1e-12


def test_jacobian_voxel_size_and_sampled_vs_reference():
    f3 = cu(G["jac_f3"])
    got = nb.grid_jacobian(f3, bound="dct2", voxel_size=[1.5, 2.0, 0.5], type="disp", add_identity=False)
    assert relerr(got.cpu().numpy(), G["jac3_vs"]) < 1e-12
    got = nb.grid_jacobian(f3, sample=cu(G["jac_sample"]), bound="dft", type="disp")
    assert relerr(got.cpu().numpy(), G["jac3_sampled"]) < 1e-12
    det = nb.grid_jacdet(f3, sample=cu(G["jac_sample"]), bound="dft", type="disp")
    assert relerr(det.cpu().numpy(), np.linalg.det(G["jac3_sampled"])) < 1e-10


@pytest.mark.parametrize("bound", ["dft", "dct2", "dst1", "zero"])
def test_jacobian_gradcheck(bound):
    g = torch.Generator().manual_seed(3)
    f = torch.randn((1, 4, 3, 5, 3), generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    assert gradcheck(lambda x: nb.grid_jacobian(x, bound=bound, voxel_size=[1.0, 2.0, 0.5]), (f,),
                     nondet_tol=1e-12)
    assert gradcheck(lambda x: nb.grid_jacdet(x, bound=bound, type="disp"), (f,), nondet_tol=1e-12)
    f2 = torch.randn((2, 5, 4, 2), generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    assert gradcheck(lambda x: nb.grid_jacdet(x, bound=bound), (f2,), nondet_tol=1e-12)


def test_sampled_jacdet_gradcheck():
    g = torch.Generator().manual_seed(4)
    f = torch.randn((1, 4, 4, 4, 3), generator=g, dtype=torch.float64).cuda().requires_grad_(True)
    s = (torch.rand((1, 3, 2, 3, 3), generator=g, dtype=torch.float64) * 3).cuda()
    assert gradcheck(lambda x: nb.grid_jacdet(x, sample=s, type="disp"), (f,), nondet_tol=1e-12)


def _resize_grid(inshape, factor, anchor):
    """The resize sampling grid as nitorch/spatial/_grid.py:690-734 builds it
    (restated for the test), float64 numpy (1, *outshape, D)."""
    lin = []
    for i in inshape:
        o = max(1, int(i * factor))
        a = anchor if (i > 1 and o > 1) else "e"
        if a == "c":
            lin.append(np.linspace(0, i - 1, o))
        elif a == "e":
            sc = i / o
            lin.append(np.arange(o) * sc + 0.5 * (sc - 1))
        elif a == "f":
            lin.append(np.arange(o) / factor)
        else:
            lin.append(np.arange(o) / factor + ((i - 1) - (o - 1) / factor))
    return np.stack(np.meshgrid(*lin, indexing="ij"), -1)[None]


@pytest.mark.parametrize("anchor", ["c", "e", "f", "l"])
def test_resize_vs_reference(anchor):
    x = cu(G["resize_x"])
    for k, fct in enumerate((2.0, 0.5, 1.7)):
        got = nb.resize(x, factor=fct, anchor=anchor, interpolation=3, bound="dct2").cpu().numpy()
        ref = G[f"resize_{anchor}_{k}"]
        assert got.shape == ref.shape
        # cubic resize prefilters: the reference's vendored prefilter carries
        # rounding noise (float32 scalars in its initial / final conditions),
        # largest next to the last voxel, where the 'f' / 'l' anchors sample
        # (up to 4.7e-7 relative against the exact FP64 oracle); this
        # library matches the exact oracle
        assert relerr(got, ref) < 1e-6
        grid = _resize_grid(x.shape[2:], fct, anchor)
        exact = O.grid_pull(O.spline_coeff_nd(G["resize_x"], [3], [3], dim=3), grid, [2], [3], 0)
        assert relerr(got, exact) < 1e-11


def test_resize_shape_and_affine_vs_reference():
    x = cu(G["resize_x"])
    got = nb.resize(x, shape=(5, 11, 6), interpolation=1, bound="dct2").cpu().numpy()
    assert relerr(got, G["resize_shape"]) < 1e-10
    img, aff = nb.resize(x, factor=1.5, affine=cu(G["resize_aff_in"]), anchor="c", interpolation=1, bound="dct2")
    assert relerr(img.cpu().numpy(), G["resize_aff_img"]) < 1e-10
    assert relerr(aff.cpu().numpy(), G["resize_aff_out"]) < 1e-12


def test_reslice_vs_reference():
    got = nb.reslice(cu(G["reslice_x"]), cu(G["reslice_from"]), cu(G["reslice_to"]), (7, 8, 9)).cpu().numpy()
    assert relerr(got, G["reslice_out"]) < 1e-10


def test_svf_exp_vs_reference():
    v, w = cu(G["exp_v"]), cu(G["exp_w"])
    assert relerr(svf.exp(v).cpu().numpy(), G["exp_fwd"]) < 1e-10
    assert relerr(svf.exp(v, inverse=True, displacement=True).cpu().numpy(), G["exp_inv_disp"]) < 1e-10
    vr = v.clone().requires_grad_(True)
    (svf.exp(vr) * w).sum().backward()
    assert relerr(vr.grad.cpu().numpy(), G["exp_grad"]) < 1e-9
