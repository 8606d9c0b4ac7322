"""Field and grid regularisers on the CUDA kernel (pp_regulariser /
pp_regulariser_grid through nitorch_b200.solve, the counterpart of
nitorch._C.solve): against the reference's own outputs
(tests/golden/regulariser_golden.npz, float64, 1e-12 relative) with the
wrappers' arguments, and against the FP64 oracle on larger seeded inputs
(float64 1e-12, float32 1e-5 relative to the output's max), with strided
views, batches whose weights / Hessians differ per item, and the edge
cases (all penalties zero, weights with bending, overlapping output)."""
import os

import numpy as np
import pytest
import torch

from nitorch_b200 import solve
from oracle import oracle as O
from tests._gpu_ops import relerr
from tests.test_golden_regulariser import BOUNDS, CODES, FIELD, GRID, VS

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "regulariser_golden.npz"))


def _t(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


def _np(t):
    return t.detach().double().cpu().numpy()


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_field_matches_reference_fixtures(dim):
    x = _t(GOLD[f"f{dim}_x"])
    for kb, bnd in enumerate(BOUNDS):
        bnd = bnd if isinstance(bnd, str) else bnd[:dim]
        for kp, (a, m, b, f) in enumerate(FIELD):
            got = solve.c_regulariser(x, None, None, dim, a, m, b, f, VS[:dim], bnd)
            assert relerr(_np(got), GOLD[f"f{dim}_b{kb}_p{kp}"]) < 1e-12, (kb, kp)
    for kw in range(2):
        w = _t(GOLD[f"f{dim}_w{kw}"])
        for kp, (a, m) in enumerate((([0.2], [1.0, 0.5]), ([0.3], [0.0]))):
            got = solve.c_regulariser(x[:1], w, None, dim, a, m, [0.0], [1.0], VS[:dim], "dct2")
            assert relerr(_np(got), GOLD[f"f{dim}_w{kw}_p{kp}"]) < 1e-12, (kw, kp)
    if dim > 1:
        x3 = _t(GOLD[f"f{dim}_x3"])
        for CC in (1, 3, 5, 6):
            got = solve.c_regulariser(x3, None, _t(GOLD[f"f{dim}_h{CC}"]), dim, [0.1], [0.5], [0.0], [1.0],
                                      VS[:dim], "dft")
            assert relerr(_np(got), GOLD[f"f{dim}_h{CC}_out"]) < 1e-12, CC


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_grid_matches_reference_fixtures(dim):
    v = _t(GOLD[f"g{dim}_x"])
    for kb, bnd in enumerate(BOUNDS):
        bnd = bnd if isinstance(bnd, str) else bnd[:dim]
        for kp, (a, m, b, lame, f) in enumerate(GRID):
            got = solve.c_regulariser_grid(v, None, None, a, m, b, lame, f, VS[:dim], bnd)
            assert relerr(_np(got), GOLD[f"g{dim}_b{kb}_p{kp}"]) < 1e-12, (kb, kp)
    w = _t(GOLD[f"g{dim}_w"])
    for kp, (a, m) in enumerate(((0.2, 1.0), (0.3, 0.0))):
        got = solve.c_regulariser_grid(v, w, None, a, m, 0.0, 0.0, 1.0, VS[:dim], "dft")
        assert relerr(_np(got), GOLD[f"g{dim}_w_p{kp}"]) < 1e-12, kp
    if dim > 1:
        for DD in sorted({1, dim, dim * (dim + 1) // 2}):
            got = solve.c_regulariser_grid(v[:1], None, _t(GOLD[f"g{dim}_h{DD}"]), 0.1, 0.5, 0.0, 0.0, 1.0,
                                           VS[:dim], "dct2")
            assert relerr(_np(got), GOLD[f"g{dim}_h{DD}_out"]) < 1e-12, DD


def _rand(shape, seed, lo=None):
    g = np.random.default_rng(seed)
    return g.random(shape) + lo if lo is not None else g.standard_normal(shape)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("bound", ["dct2", "dft", "dst2", "replicate", "zero"])
def test_field_vs_oracle_larger(dtype, bound):
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    x = _rand((2, 3, 33, 30, 29), 1)
    xc = _t(x, dtype)
    for (a, m, b) in (([0.1, 0.2, 0.3], [1.0, 0.5, 2.0], [0.0]), ([0.01], [0.1], [1.0, 0.5, 0.2])):
        got = solve.c_regulariser(xc, None, None, 3, a, m, b, 1.0, [1.2, 0.9, 1.5], bound)
        ref = O.regulariser(x, None, None, a, m, b, [1.2, 0.9, 1.5], [CODES[bound]])
        assert relerr(_np(got), ref) < tol, (a, m, b)
    # weights and a symmetric Hessian that differ per batch item
    w = _rand((2, 1, 33, 30, 29), 2, lo=0.5)
    got = solve.c_regulariser(xc, _t(w, dtype), None, 3, [0.2], [1.0], [0.0], 1.0, [1.0], bound)
    assert relerr(_np(got), O.regulariser(x, w, None, [0.2], [1.0], [0.0], [1.0], [CODES[bound]])) < tol
    h = _rand((2, 6, 33, 30, 29), 3, lo=0.0)
    got = solve.c_regulariser(xc, None, _t(h, dtype), 3, [0.2], [1.0], [0.0], 1.0, [1.0], bound)
    assert relerr(_np(got), O.regulariser(x, None, h, [0.2], [1.0], [0.0], [1.0], [CODES[bound]])) < tol


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("bound", ["dft", "dct2", "dst1", "zero"])
def test_grid_vs_oracle_larger_and_strided(dtype, bound):
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    v = _rand((2, 31, 28, 26, 3), 4)
    # components first in memory (a movedim view): any strides
    vc = _t(np.moveaxis(v, -1, 1), dtype).movedim(1, -1)
    for (a, m, b, lame) in ((0.1, 1.0, 0.0, (0.0, 0.0)), (0.01, 0.2, 0.5, (0.7, 0.4)), (0.0, 0.0, 0.0, (1.0, 2.0))):
        got = solve.c_regulariser_grid(vc, None, None, a, m, b, lame, 1.0, [1.2, 0.9, 1.5], bound)
        ref = np.moveaxis(O.regulariser_grid(np.moveaxis(v, -1, 1), None, None, a, m, b, lame[0], lame[1],
                                             [1.2, 0.9, 1.5], [CODES[bound]]), 1, -1)
        assert relerr(_np(got), ref) < tol, (a, m, b, lame)
    w = _rand((2, 31, 28, 26), 5, lo=0.5)
    h = _rand((2, 31, 28, 26, 6), 6, lo=0.0)
    got = solve.c_regulariser_grid(vc, _t(w, dtype), None, 0.2, 1.0, 0.0, 0.0, 1.0, [1.0], bound)
    ref = O.regulariser_grid(np.moveaxis(v, -1, 1), w, None, 0.2, 1.0, 0.0, 0.0, 0.0, [1.0], [CODES[bound]])
    assert relerr(_np(got), np.moveaxis(ref, 1, -1)) < tol
    got = solve.c_regulariser_grid(vc, None, _t(h, dtype), 0.2, 1.0, 0.0, 0.0, 1.0, [1.0], bound)
    ref = O.regulariser_grid(np.moveaxis(v, -1, 1), None, np.moveaxis(h, -1, 1), 0.2, 1.0, 0.0, 0.0, 0.0, [1.0],
                             [CODES[bound]])
    assert relerr(_np(got), np.moveaxis(ref, 1, -1)) < tol


def test_edge_cases():
    x = _t(_rand((1, 2, 8, 7, 6), 7))
    # every penalty zero: the Hessian product alone (zeros without one)
    h = _t(_rand((1, 2, 8, 7, 6), 8, lo=0.0))
    assert torch.equal(solve.c_regulariser(x, None, None, 3), torch.zeros_like(x))
    assert relerr(_np(solve.c_regulariser(x, None, h, 3)), _np(h * x)) < 1e-15
    with pytest.raises(ValueError):
        solve.c_regulariser(x, torch.ones_like(x), None, 3, 0.1, 1.0, 1.0)
    with pytest.raises(ValueError):
        solve.c_regulariser_grid(x[:, 0, ..., None].expand(1, 8, 7, 6, 3).contiguous(),
                                 torch.ones(1, 8, 7, 6, dtype=x.dtype, device="cuda"), None, 0.1, 1.0, lame=(1.0, 0.0))
    with pytest.raises(RuntimeError):  # output overlapping the input
        solve.c_regulariser(x, None, None, 3, 0.1, 1.0, output=x)
    # unbatched inputs with `dim`: leading dimensions added and removed
    y = solve.c_regulariser(x[0], None, None, 3, 0.1, 1.0)
    assert y.shape == x[0].shape
    assert relerr(_np(y), O.regulariser(_np(x), None, None, [0.1], [1.0], [0.0], [1.0], [2])[0]) < 1e-12
