"""The multigrid resampling oracle (native fmg_prolongation / fmg_restriction,
native resize with its modes, adjoint and normalisation, the multigrid
solvers' prolong / restrict) against the reference's own outputs
(tests/golden/multires_golden.npz, made by make_golden.py multires).
float64, 1e-12 relative."""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "multires_golden.npz"))
BOUNDS = (0, 1, 2, 3, 4, 5, 7)


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("b", BOUNDS)
def test_fmg_oracle_vs_reference(k, b):
    x = GOLD[f"fmg_x{k}"]
    _close(O.fmg_prolongation(x, [b]), GOLD[f"fmg_pro{k}_b{b}"])
    _close(O.fmg_restriction(x, [b]), GOLD[f"fmg_res{k}_b{b}"])


@pytest.mark.parametrize("mode", range(4))
@pytest.mark.parametrize("adj", (0, 1))
@pytest.mark.parametrize("norm", (0, 1))
@pytest.mark.parametrize("kf", (0, 1))
@pytest.mark.parametrize("order", (1, 3))
def test_native_resize_oracle_vs_reference(mode, adj, norm, kf, order):
    fac = (2.0, 0.7)[kf]
    got = O.resize_native(GOLD["rz_x"], None, [fac], [2], [order], [mode], bool(adj), bool(norm))
    _close(got, GOLD[f"rz_m{mode}_a{adj}_n{norm}_f{kf}_o{order}"])


def test_native_wrappers_vs_reference():
    """prolongation / restriction and their backward (nitorch/_C/src/
    resize.cpp:63-128): the native resize at factor 1, edge alignment,
    quadratic / linear, on the lattice of the given output."""
    x, xf = GOLD["rz_x"], GOLD["wrap_fine"]
    _close(O.resize_native(x, (10, 12, 14), [1.0], [2], [2], [0], False, False), GOLD["wrap_prolongation"])
    _close(O.resize_native(xf, (5, 6, 7), [1.0], [2], [2], [0], True, False), GOLD["wrap_prolongation_backward"])
    _close(O.resize_native(xf, (5, 6, 7), [1.0], [2], [1], [0], True, True), GOLD["wrap_restriction"])
    _close(O.resize_native(x, (10, 12, 14), [1.0], [2], [1], [0], False, True), GOLD["wrap_restriction_backward"])


def _grid_factors(inp_moved, out_last):
    """The channel factors of nitorch/_C/resize.py:176,212: out / in over
    the LAST `dim` axes of the channel-first input and of the channel-last
    output (so (Y'/X, Z'/Y, D/Z) in 3-D: the reference takes them after
    moving the output back)."""
    dim = out_last.shape[-1]
    return np.array([o / i for i, o in zip(inp_moved.shape[-dim:], out_last.shape[-dim:])])


def test_python_wrappers_vs_reference():
    """nitorch/_C/resize.py:99-215 over the fmg operators: factor / shape
    forms and the displacement-grid forms."""
    x, xf = GOLD["rz_x"], GOLD["wrap_fine"]
    _close(O.fmg_prolongation(x, [1]), GOLD["c_prolongation"])
    _close(O.fmg_restriction(xf, [5]), GOLD["c_restriction"])
    _close(O.fmg_restriction(xf, [2], shape=(4, 7, 5)), GOLD["c_restriction_shape"])
    v, vf = GOLD["grid_coarse"], GOLD["grid_fine"]
    vm, vfm = np.moveaxis(v, -1, 1), np.moveaxis(vf, -1, 1)
    pg = np.moveaxis(O.fmg_prolongation(vm, [2]), 1, -1)
    _close(pg * _grid_factors(vm, pg), GOLD["c_prolongation_grid"])
    rg = np.moveaxis(O.fmg_restriction(vfm, [2]), 1, -1)
    _close(rg * _grid_factors(vfm, rg), GOLD["c_restriction_grid"])


def test_solver_prolong_restrict_vs_reference():
    v, vf = GOLD["grid_coarse"], GOLD["grid_fine"]
    _close(O.solver_prolong(v), GOLD["sv_prolong"], 1e-10)
    _close(O.solver_prolong(v, bound=5, order=3), GOLD["sv_prolong_o3"], 1e-10)
    _close(O.solver_restrict(vf), GOLD["sv_restrict"], 1e-10)
    _close(O.solver_restrict(vf, shape=(4, 5, 8)), GOLD["sv_restrict_shape"], 1e-10)
    _close(O.solver_prolong(v[:1])[0], GOLD["sv_prolong_nobatch"], 1e-10)
