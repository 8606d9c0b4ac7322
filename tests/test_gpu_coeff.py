"""CUDA prefilter vs the reference's vendored prefilter (golden fixtures)
and vs the FP64 oracle; interpolation property; in-place and strided use.
Tolerances: float64 vs golden 2e-7 relative (the vendored reference's own
rounding noise, defect D7); float64 vs FP64 oracle 1e-11; float32 vs FP64
oracle 1e-5 relative."""
import os

import numpy as np
import pytest
import torch

import nitorch_b200 as nb
from nitorch_b200 import coeff
from oracle import oracle as O
from tests._gpu_ops import relerr

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CO = np.load(os.path.join(G, "coeff_golden.npz"))


@pytest.mark.parametrize("order", range(2, 8))
@pytest.mark.parametrize("bound", [2, 3, 6])
@pytest.mark.parametrize("n", [2, 3, 7, 40])
def test_coeff_vs_golden_and_oracle(order, bound, n):
    k = f"o{order}_b{bound}_n{n}"
    x = torch.from_numpy(CO[k + "_x"]).cuda()
    y = coeff.spline_coeff(x, bound, order, dim=-1).cpu().numpy()
    assert relerr(y, CO[k + "_y"]) < 2e-7
    assert relerr(y, O.spline_coeff(CO[k + "_x"], bound, order)) < 1e-11
    y32 = coeff.spline_coeff(x.float(), bound, order, dim=-1).double().cpu().numpy()
    assert relerr(y32, O.spline_coeff(CO[k + "_x"], bound, order)) < 1e-5


@pytest.mark.parametrize("order", [2, 3, 5, 7])
def test_coeff_nd_golden(order):
    x = torch.from_numpy(CO[f"nd_o{order}_x"]).cuda()
    y = coeff.spline_coeff_nd(x, [3], [order], dim=3).cpu().numpy()
    assert relerr(y, CO[f"nd_o{order}_y"]) < 2e-7


@pytest.mark.parametrize("bound", [("dct1", 2), ("dct2", 3), ("dft", 6), ("zero", 0), ("replicate", 1)])
@pytest.mark.parametrize("shape", [(17, 33, 9), (64, 1, 40), (200, 3, 5)])
def test_coeff_axes_and_layouts(bound, shape):
    name, bts = bound
    r = np.random.default_rng(len(shape))
    x = r.standard_normal((2,) + shape)
    ref = O.spline_coeff_nd(x, [bts], [3], dim=3)
    X = torch.from_numpy(x).cuda()
    assert relerr(coeff.spline_coeff_nd(X, [bts], [3], dim=3).cpu().numpy(), ref) < 1e-11
    Xt = X.transpose(1, 3).contiguous().transpose(1, 3)    # non-contiguous storage
    assert relerr(coeff.spline_coeff_nd(Xt, [bts], [3], dim=3).cpu().numpy(), ref) < 1e-11
    Xi = X.clone()
    out = coeff.spline_coeff_nd(Xi, [bts], [3], dim=3, inplace=True)
    assert out.data_ptr() == Xi.data_ptr()
    assert relerr(Xi.cpu().numpy(), ref) < 1e-11
    assert relerr(nb.spline_coeff_nd(X.float(), 3, name, dim=3).double().cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32, torch.bfloat16])
@pytest.mark.parametrize("n", [8, 9, 15, 16, 17, 24, 25, 96, 129, 192, 256, 384, 388, 500])
@pytest.mark.parametrize("bound", [2, 3, 6])
def test_coeff_register_chunk_lengths(dtype, n, bound):
    """Line lengths around the recursions' register chunks, tiles at the 48 KB
    default shared-memory limit (96 / 192 / 384 samples), either side of the
    longest full tile (387 samples) and in the long-line kernel (500), along
    the fastest axis (warps stage whole lines) and a strided one (threads
    stage groups of adjacent lines), with full and partial last tiles."""
    r = np.random.default_rng(n + bound)
    tol = {torch.float64: 1e-11, torch.float32: 1e-5, torch.bfloat16: 1e-5}[dtype]
    for order in (3, 7):
        for shape, axis in (((3, 5, n), -1), ((3, n, 37), 1), ((140, n), -1), ((n, 140), 0)):
            x = torch.from_numpy(r.standard_normal(shape)).to(dtype)
            ref = O.spline_coeff(x.double().numpy(), bound, order, dim=axis)
            y = coeff.spline_coeff(x.cuda(), bound, order, dim=axis)
            if dtype == torch.bfloat16:
                # recursions in float, one bfloat16 rounding of the output
                assert relerr(y.double().cpu().numpy(), ref) < 8e-3
            else:
                assert relerr(y.double().cpu().numpy(), ref) < tol


@pytest.mark.parametrize("dtype,n", [(torch.float32, 30000), (torch.float32, 60000), (torch.float64, 30000)])
def test_coeff_lines_beyond_tile_budget(dtype, n):
    """Lines too long for two CTAs per SM (one wide tile per CTA), and lines
    too long for shared memory altogether (recursion in global memory)."""
    r = np.random.default_rng(n)
    x = r.standard_normal((3, n))
    ref = O.spline_coeff(x, 3, 3, dim=-1)
    y = coeff.spline_coeff(torch.from_numpy(x).to(dtype).cuda(), 3, 3, dim=-1)
    assert relerr(y.double().cpu().numpy(), ref) < (1e-11 if dtype == torch.float64 else 1e-5)


def test_coeff_bf16_line_too_long_raises():
    with pytest.raises(Exception):
        coeff.spline_coeff(torch.zeros(2, 60000, device="cuda", dtype=torch.bfloat16), 3, 3, dim=-1)


def test_coeff_interpolates_long_lines():
    x = torch.randn(1, 1, 96, 80, 72, dtype=torch.double, device="cuda")
    grid = nb.identity_grid(x.shape[2:], dtype=torch.double, device="cuda")[None]
    for order in (2, 3, 5, 7):
        y = nb.grid_pull(x, grid, order, "dct2", True, prefilter=True)
        assert (y - x).abs().max().item() < 1e-9


def test_coeff_unsupported_bound_raises():
    x = torch.randn(4, 5, device="cuda")
    with pytest.raises(NotImplementedError):
        coeff.spline_coeff(x, 4, 3)
    # order 0 / 1 are the identity whatever the bound (coeff.py:302-305)
    assert torch.equal(coeff.spline_coeff(x, 4, 1), x)


def test_coeff_bf16_storage():
    x = torch.randn(2, 40, 33, 20, device="cuda").bfloat16()
    ref = O.spline_coeff_nd(x.double().cpu().numpy(), [3], [3], dim=3)
    y = coeff.spline_coeff_nd(x, [3], [3], dim=3)
    assert y.dtype == torch.bfloat16
    # three passes, each stored in bfloat16
    assert relerr(y.double().cpu().numpy(), ref) < 3 * 2.0 ** -8
