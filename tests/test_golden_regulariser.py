"""The regulariser oracle (field and grid, every penalty mix, weights,
Hessian layouts, 1-3-D, seven bounds) against the reference's own outputs
through its wrappers nitorch/_C/solve.py c_regulariser / c_regulariser_grid
(tests/golden/regulariser_golden.npz, made by make_golden.py regulariser).
float64, 1e-12 relative."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "regulariser_golden.npz"))
CODES = {"replicate": 0, "dct1": 1, "dct2": 2, "dst1": 3, "dst2": 4, "dft": 5, "zero": 7}
# the cases of make_golden.py (REG_FIELD, REG_GRID, REG_BOUNDS, REG_VS)
FIELD = [([0.1], [0.0], [0.0], [1.0]), ([0.1], [1.0, 2.0], [0.0], [1.0, 0.5]),
         ([0.05], [0.3], [0.7, 0.2], [1.0]), ([0.0], [0.0], [1.0], [2.0])]
GRID = [(0.1, 0.0, 0.0, (0.0, 0.0), 1.0), (0.1, 1.0, 0.0, (0.0, 0.0), 1.0), (0.05, 0.3, 0.7, (0.0, 0.0), 2.0),
        (0.02, 0.4, 0.0, (0.6, 0.3), 1.0), (0.01, 0.2, 0.5, (0.7, 0.4), 0.5), (0.0, 0.0, 0.0, (1.0, 0.0), 1.0),
        (0.0, 0.0, 0.0, (0.0, 1.0), 1.0)]
BOUNDS = ["dct2", "dft", "zero", "dst1", ["dct1", "dst2", "replicate"]]
VS = [1.3, 0.8, 1.1]


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


def _codes(bnd, dim):
    return [CODES[bnd]] if isinstance(bnd, str) else [CODES[v] for v in bnd[:dim]]


def _chan(v, C):
    return [v[min(c, len(v) - 1)] for c in range(C)]


def field(x, w, h, a, m, b, f, vs, bnd):
    """c_regulariser's argument handling (solve.py:21-78): per-channel lists
    padded with their last entry, scaled by `factor`."""
    C = x.shape[1]
    f = _chan(f, C)
    a, m, b = ([u * s for u, s in zip(_chan(v, C), f)] for v in (a, m, b))
    return O.regulariser(x, w, h, a, m, b, vs, bnd)


def grid(v, w, h, a, m, b, lame, f, vs, bnd):
    """c_regulariser_grid (solve.py:80-142): components last, scalar
    penalties scaled by `factor`, lame = (shear, div)."""
    x = np.moveaxis(v, -1, 1)
    hh = None if h is None else np.moveaxis(h, -1, 1)
    y = O.regulariser_grid(x, w, hh, a * f, m * f, b * f, lame[0] * f, lame[1] * f, vs, bnd)
    return np.moveaxis(y, 1, -1)


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("kb", range(len(BOUNDS)))
def test_field_regulariser_oracle_vs_reference(dim, kb):
    x = GOLD[f"f{dim}_x"]
    for kp, (a, m, b, f) in enumerate(FIELD):
        _close(field(x, None, None, a, m, b, f, VS[:dim], _codes(BOUNDS[kb], dim)), GOLD[f"f{dim}_b{kb}_p{kp}"])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_field_regulariser_weights_and_hessian(dim):
    x = GOLD[f"f{dim}_x"]
    for kw in range(2):
        w = GOLD[f"f{dim}_w{kw}"]
        for kp, (a, m) in enumerate((([0.2], [1.0, 0.5]), ([0.3], [0.0]))):
            _close(field(x[:1], w, None, a, m, [0.0], [1.0], VS[:dim], [2]), GOLD[f"f{dim}_w{kw}_p{kp}"])
    if dim > 1:
        x3 = GOLD[f"f{dim}_x3"]
        for CC in (1, 3, 5, 6):
            _close(field(x3, None, GOLD[f"f{dim}_h{CC}"], [0.1], [0.5], [0.0], [1.0], VS[:dim], [5]),
                   GOLD[f"f{dim}_h{CC}_out"])


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("kb", range(len(BOUNDS)))
def test_grid_regulariser_oracle_vs_reference(dim, kb):
    v = GOLD[f"g{dim}_x"]
    for kp, (a, m, b, lame, f) in enumerate(GRID):
        _close(grid(v, None, None, a, m, b, lame, f, VS[:dim], _codes(BOUNDS[kb], dim)), GOLD[f"g{dim}_b{kb}_p{kp}"])


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_grid_regulariser_weights_and_hessian(dim):
    v = GOLD[f"g{dim}_x"]
    w = GOLD[f"g{dim}_w"]
    for kp, (a, m) in enumerate(((0.2, 1.0), (0.3, 0.0))):
        _close(grid(v, w, None, a, m, 0.0, (0.0, 0.0), 1.0, VS[:dim], [5]), GOLD[f"g{dim}_w_p{kp}"])
    if dim > 1:
        for DD in sorted({1, dim, dim * (dim + 1) // 2}):
            _close(grid(v[:1], None, GOLD[f"g{dim}_h{DD}"], 0.1, 0.5, 0.0, (0.0, 0.0), 1.0, VS[:dim], [2]),
                   GOLD[f"g{dim}_h{DD}_out"])


def test_bending_with_weights_is_an_error():
    x = GOLD["f3_x"][:1]
    with pytest.raises(ValueError):
        O.regulariser(x, np.ones_like(x), None, [0.1], [1.0], [1.0])
    with pytest.raises(ValueError):
        O.regulariser_grid(np.moveaxis(GOLD["g3_x"], -1, 1), GOLD["g3_w"], None, 0.1, 1.0, 0.0, 0.5, 0.0)
