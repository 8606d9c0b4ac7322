"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a checkout where the reference is available:
    python oracle/build_ref.py            # compiles nitorch/_C into oracle/_ref
    python tests/golden/make_golden.py

Writes
  pushpull_golden.npz : seeded small inputs and the compiled reference's
                        outputs of its eight push/pull functions, float64,
                        1/2/3-D, seven bounds, orders 0-7; float32 order-0
                        cases for the bit-exact checks.
  coeff_golden.npz    : outputs of the reference's vendored prefilter
                        (nitorch/_C/_ts/coeff.py) for orders 2-7, bounds
                        dct1 / dct2 / dft, several line lengths, plus 3-D
                        spline_coeff_nd volumes.
  config1_golden.npz  : checksums of the reference's pull / push on the
                        seeded config-1 workload (1x1x64^3, order 1, dct2).
  multires_golden.npz : outputs of the reference's multigrid resampling
                        (native fmg_prolongation / fmg_restriction, native
                        resize with modes / adjoint / normalisation, the
                        prolongation / restriction wrappers, the multigrid
                        solvers' prolong / restrict) on seeded float64
                        inputs (`python tests/golden/make_golden.py multires`).
  spatial_golden.npz  : outputs of the reference's nitorch.spatial callers of
                        the path (grid_jacobian / grid_jacdet, resize,
                        reslice, exp of a velocity field and its autograd
                        gradient) on seeded float64 inputs.
                        (`python tests/golden/make_golden.py spatial` writes
                        this file alone.)
  regulariser_golden.npz : outputs of the reference's field and grid
                        regularisers (nitorch/_C/solve.py) on seeded float64
                        inputs (`python tests/golden/make_golden.py
                        regulariser`).

Reference defects are handled as in tests/test_oracle_vs_reference.py: the
grid_grad_backward target is laid out with a last-dimension stride > 1 (D2),
and 1-D grid_grad is generated with extrapolation on (D6).  Orders 5-7 of
grid_grad_backward carry defect D3 (zero second derivatives); those grid
gradients are stored under a "_d3" key.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reference as R  # noqa: E402
from tests._cases import BOUND_CODES, ORDERS, make_case, config1_inputs  # noqa: E402


def _t(a, rg=False):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.requires_grad_(rg) if rg else t


def _strided_last(a):
    n, c, k = a.shape[0], a.shape[1], a.shape[-1]
    sp = a.shape[2:-1]
    p = int(np.prod(sp))
    st, acc = [], 1
    for s in reversed(sp):
        st.insert(0, acc)
        acc *= s
    t = torch.empty_strided(a.shape, [c * k * p, k * p] + st + [p], dtype=torch.float64)
    t.copy_(torch.from_numpy(a))
    return t


def pushpull(ref):
    B = {v.value: v for v in ref.BoundType.__members__.values()}
    I = {v.value: v for v in ref.InterpolationType.__members__.values()}
    out = {}
    for dim in (1, 2, 3):
        for bound in BOUND_CODES:
            for order in ORDERS:
                key = f"d{dim}_b{bound}_o{order}"
                vol, grid = make_case(dim, seed=7000 + 100 * dim + 10 * bound + order,
                                      in_size=5 if dim < 3 else 4, out_size=4 if dim < 3 else 3)
                g = np.random.default_rng(8000 + 100 * dim + 10 * bound + order)
                tgt = g.standard_normal((1, vol.shape[1]) + grid.shape[1:-1])
                gpush = g.standard_normal(vol.shape)
                gcount = g.standard_normal((1, 1) + vol.shape[2:])
                ggrad = g.standard_normal((1, vol.shape[1]) + grid.shape[1:-1] + (dim,))
                b, o = [B[bound]], [I[order]]
                ex = 1
                out[key + "_vol"] = vol
                out[key + "_grid"] = grid
                out[key + "_tgt"] = tgt
                out[key + "_gpush"] = gpush
                out[key + "_gcount"] = gcount
                out[key + "_ggrad"] = ggrad
                out[key + "_pull"] = ref.grid_pull(_t(vol), _t(grid), b, o, ex).numpy()
                out[key + "_sgrad"] = ref.grid_grad(_t(vol), _t(grid), b, o, ex).numpy()
                out[key + "_push"] = ref.grid_push(_t(tgt), _t(grid), list(vol.shape[2:]), b, o, ex).numpy()
                out[key + "_count"] = ref.grid_count(_t(grid), list(vol.shape[2:]), b, o, ex).numpy()
                r = ref.grid_pull_backward(_t(tgt), _t(vol, True), _t(grid, True), b, o, ex)
                out[key + "_pullbwd_in"] = r[0].detach().numpy()
                out[key + "_pullbwd_grid"] = r[1].detach().numpy()
                r = ref.grid_push_backward(_t(gpush), _t(tgt, True), _t(grid, True), b, o, ex)
                out[key + "_pushbwd_in"] = r[0].detach().numpy()
                out[key + "_pushbwd_grid"] = r[1].detach().numpy()
                r = ref.grid_count_backward(_t(gcount), _t(grid, True), b, o, ex)
                out[key + "_countbwd_grid"] = r.detach().numpy()
                r = ref.grid_grad_backward(_strided_last(ggrad), _t(vol, True), _t(grid, True), b, o, ex)
                out[key + "_gradbwd_in"] = r[0].detach().numpy()
                out[key + ("_gradbwd_grid_d3" if order >= 5 else "_gradbwd_grid")] = r[1].detach().numpy()
    # float32 order-0 cases, no extrapolation (OOB mask) and both tolerances
    for dim in (1, 2, 3):
        for bound in BOUND_CODES:
            vol, grid = make_case(dim, seed=9000 + 10 * dim + bound, spread=3.0)
            vol = vol.astype(np.float32)
            grid = grid.astype(np.float32)
            key = f"f32_d{dim}_b{bound}"
            out[key + "_vol"] = vol
            out[key + "_grid"] = grid
            for ex in (0, 1, 2):
                out[key + f"_pull_ex{ex}"] = ref.grid_pull(_t(vol), _t(grid), [B[bound]], [I[0]], ex).numpy()
    return out


def coeff(ts):
    out = {}
    r = np.random.default_rng(4242)
    for order in range(2, 8):
        for bound in (2, 3, 6):
            for n in (2, 3, 7, 40):
                x = r.standard_normal((3, n))
                y = ts.spline_coeff(torch.from_numpy(x.copy()), bound, order, dim=-1).numpy()
                out[f"o{order}_b{bound}_n{n}_x"] = x
                out[f"o{order}_b{bound}_n{n}_y"] = y
    for order in (2, 3, 5, 7):
        x = r.standard_normal((2, 6, 5, 7))
        y = ts.spline_coeff_nd(torch.from_numpy(x.copy()), [3], [order], dim=3).numpy()
        out[f"nd_o{order}_x"] = x
        out[f"nd_o{order}_y"] = y
    return out


def config1(ref):
    x, grid, y = config1_inputs()
    B, I = ref.BoundType.dct2, ref.InterpolationType.linear
    tx, tg, ty = (torch.from_numpy(a) for a in (x, grid, y))
    out = {}
    p = ref.grid_pull(tx, tg, [B], [I], 0)
    q = ref.grid_push(ty, tg, list(x.shape[2:]), [B], [I], 0)
    out["pull_sum"] = p.sum().item()
    out["pull_sumsq"] = (p * p).sum().item()
    out["push_sum"] = q.sum().item()
    out["push_sumsq"] = (q * q).sum().item()
    out["inner_pull_y"] = (p * ty).sum().item()
    out["inner_x_push"] = (tx * q).sum().item()
    out["pull_slice"] = p[0, 0, 32].numpy()
    out["push_slice"] = q[0, 0, 32].numpy()
    return {k: np.asarray(v) for k, v in out.items()}


def spatial(S):
    """nitorch.spatial callers of the push/pull path, float64."""
    out = {}
    g = torch.Generator().manual_seed(77)
    # Jacobians by central differences, all bounds, both field types
    f3 = torch.randn((1, 7, 6, 5, 3), generator=g, dtype=torch.float64)
    f2 = torch.randn((1, 8, 9, 2), generator=g, dtype=torch.float64)
    f1s = torch.randn((1, 6, 1, 5, 3), generator=g, dtype=torch.float64)  # a singleton axis
    out["jac_f3"], out["jac_f2"], out["jac_f1s"] = f3.numpy(), f2.numpy(), f1s.numpy()
    for b in ("dft", "dct2", "dct1", "dst1", "dst2", "zero", "replicate"):
        for typ in ("grid", "disp"):
            out[f"jac3_{b}_{typ}"] = S.grid_jacobian(f3, bound=b, type=typ).numpy()
            out[f"jacdet3_{b}_{typ}"] = S.grid_jacdet(f3, bound=b, type=typ).numpy()
            out[f"jac2_{b}_{typ}"] = S.grid_jacobian(f2, bound=b, type=typ).numpy()
        out[f"jac1s_{b}"] = S.grid_jacobian(f1s, bound=b, type="disp").numpy()
    out["jac3_vs"] = S.grid_jacobian(f3, bound="dct2", voxel_size=[1.5, 2.0, 0.5], type="disp",
                                     add_identity=False).numpy()
    smp = torch.rand((1, 4, 5, 3, 3), generator=g, dtype=torch.float64) * 5
    out["jac_sample"] = smp.numpy()
    out["jac3_sampled"] = S.grid_jacobian(f3, sample=smp, bound="dft", type="disp").numpy()
    # resize: anchors x factors, cubic dct2 (prefilter on by default)
    x = torch.randn((1, 2, 9, 8, 7), generator=g, dtype=torch.float64)
    out["resize_x"] = x.numpy()
    for a in ("c", "e", "f", "l"):
        for k, fct in enumerate((2.0, 0.5, 1.7)):
            out[f"resize_{a}_{k}"] = S.resize(x, factor=fct, anchor=a, interpolation=3, bound="dct2").numpy()
    out["resize_shape"] = S.resize(x, shape=(5, 11, 6), interpolation=1, bound="dct2").numpy()
    aff = torch.eye(4, dtype=torch.float64)
    aff[:3, :3] = torch.diag(torch.tensor([1.2, 0.9, 2.0], dtype=torch.float64))
    aff[:3, 3] = torch.tensor([3.0, -1.0, 0.5], dtype=torch.float64)
    rz, raff = S.resize(x, factor=1.5, affine=aff, anchor="c", interpolation=1, bound="dct2")
    out["resize_aff_in"], out["resize_aff_out"], out["resize_aff_img"] = aff.numpy(), raff.numpy(), rz.numpy()
    # reslice: linear, zero bound (defaults), shape_to given
    y = torch.randn((1, 1, 10, 9, 8), generator=g, dtype=torch.float64)
    a_from = torch.eye(4, dtype=torch.float64)
    a_from[:3, :3] *= 1.5
    a_to = torch.eye(4, dtype=torch.float64)
    a_to[:3, :3] += 0.1 * torch.randn((3, 3), generator=g, dtype=torch.float64)
    a_to[:3, 3] = torch.tensor([1.0, 2.0, -0.5], dtype=torch.float64)
    out["reslice_x"], out["reslice_from"], out["reslice_to"] = y.numpy(), a_from.numpy(), a_to.numpy()
    out["reslice_out"] = S.reslice(y, a_from, a_to, (7, 8, 9)).numpy()
    # velocity exponentiation, forward and autograd gradient
    v = torch.randn((1, 8, 9, 7, 3), generator=g, dtype=torch.float64)
    v = torch.nn.functional.avg_pool3d(v.movedim(-1, 1), 3, 1, 1).movedim(1, -1) * 3
    w = torch.randn(v.shape, generator=g, dtype=torch.float64)
    out["exp_v"], out["exp_w"] = v.numpy(), w.numpy()
    out["exp_fwd"] = S.exp(v).numpy()
    out["exp_inv_disp"] = S.exp(v, inverse=True, displacement=True).numpy()
    vr = v.clone().requires_grad_(True)
    (S.exp(vr) * w).sum().backward()
    out["exp_grad"] = vr.grad.numpy()
    return {k: np.asarray(v) for k, v in out.items()}


def multires(ref, S):
    """nitorch's multigrid resampling, float64: the native fmg_prolongation /
    fmg_restriction (3-D: the reference raises on 1-D / 2-D inputs), the
    native resize with its alignment modes, adjoint and normalisation, the
    native prolongation / restriction wrappers and their backward, the
    displacement-grid wrappers of nitorch/_C/resize.py and the multigrid
    solvers' prolong / restrict (nitorch/spatial/_solvers.py)."""
    import nitorch._C.resize as CR
    import nitorch.spatial._solvers as SV
    out = {}
    g = torch.Generator().manual_seed(91)
    BT = {0: ref.BoundType.replicate, 1: ref.BoundType.dct1, 2: ref.BoundType.dct2, 3: ref.BoundType.dst1,
          4: ref.BoundType.dst2, 5: ref.BoundType.dft, 7: ref.BoundType.zero}
    IT = [ref.InterpolationType.nearest, ref.InterpolationType.linear, ref.InterpolationType.quadratic,
          ref.InterpolationType.cubic]
    GA = [ref.GridAlignType.edge, ref.GridAlignType.center, ref.GridAlignType.first, ref.GridAlignType.last]
    shapes = [(1, 2, 5, 6, 7), (2, 1, 9, 4, 3), (1, 1, 1, 8, 3), (1, 2, 6, 6, 6)]
    for k, sh in enumerate(shapes):
        x = torch.randn(sh, generator=g, dtype=torch.float64)
        out[f"fmg_x{k}"] = x.numpy()
        for b, bt in BT.items():
            out[f"fmg_pro{k}_b{b}"] = ref.fmg_prolongation(x, torch.Tensor(), [bt]).numpy()
            out[f"fmg_res{k}_b{b}"] = ref.fmg_restriction(x, torch.Tensor(), [bt]).numpy()
    x = torch.randn((1, 2, 5, 6, 7), generator=g, dtype=torch.float64)
    out["rz_x"] = x.numpy()
    for mode in range(4):
        for adj in (0, 1):
            for norm in (0, 1):
                for kf, fac in enumerate((2.0, 0.7)):
                    for order in (1, 3):
                        key = f"rz_m{mode}_a{adj}_n{norm}_f{kf}_o{order}"
                        out[key] = ref.resize(x, torch.Tensor(), [fac], [BT[2]], [IT[order]], [GA[mode]],
                                              bool(adj), bool(norm)).numpy()
    # the native wrappers with an output lattice given
    xf = torch.randn((1, 2, 10, 12, 14), generator=g, dtype=torch.float64)
    out["wrap_fine"] = xf.numpy()
    out["wrap_prolongation"] = ref.prolongation(x, torch.zeros((1, 2, 10, 12, 14), dtype=torch.float64),
                                                [], []).numpy()
    out["wrap_prolongation_backward"] = ref.prolongation_backward(
        xf, torch.zeros((1, 2, 5, 6, 7), dtype=torch.float64), [], []).numpy()
    out["wrap_restriction"] = ref.restriction(xf, torch.zeros((1, 2, 5, 6, 7), dtype=torch.float64),
                                              [], []).numpy()
    out["wrap_restriction_backward"] = ref.restriction_backward(
        x, torch.zeros((1, 2, 10, 12, 14), dtype=torch.float64), [], []).numpy()
    # nitorch/_C/resize.py wrappers (factor / shape, displacement grids)
    out["c_prolongation"] = CR.c_prolongation(x, factor=2., bound="dct1").numpy()
    out["c_restriction"] = CR.c_restriction(xf, factor=2., bound="dft").numpy()
    out["c_restriction_shape"] = CR.c_restriction(xf, shape=(4, 7, 5)).numpy()
    v = torch.randn((1, 5, 6, 7, 3), generator=g, dtype=torch.float64)
    vf = torch.randn((1, 10, 12, 14, 3), generator=g, dtype=torch.float64)
    out["grid_coarse"], out["grid_fine"] = v.numpy(), vf.numpy()
    out["c_prolongation_grid"] = CR.c_prolongation_grid(v.clone()).numpy()
    out["c_restriction_grid"] = CR.c_restriction_grid(vf.clone()).numpy()
    # multigrid solvers' prolong / restrict (channel-last)
    out["sv_prolong"] = SV.prolong(v.clone(), dim=3).numpy()
    out["sv_prolong_o3"] = SV.prolong(v.clone(), order=3, bound="dft", dim=3).numpy()
    out["sv_restrict"] = SV.restrict(vf.clone(), dim=3).numpy()
    out["sv_restrict_shape"] = SV.restrict(vf.clone(), shape=(4, 5, 8), dim=3).numpy()
    out["sv_prolong_nobatch"] = SV.prolong(v[0].clone()).numpy()  # (*spatial, K): dim = 3 by default
    return {k: np.asarray(v) for k, v in out.items()}


REG_FIELD = [  # (absolute, membrane, bending, factor)
    ([0.1], [0.0], [0.0], [1.0]),
    ([0.1], [1.0, 2.0], [0.0], [1.0, 0.5]),
    ([0.05], [0.3], [0.7, 0.2], [1.0]),
    ([0.0], [0.0], [1.0], [2.0]),
]
REG_GRID = [  # (absolute, membrane, bending, (shear, div), factor)
    (0.1, 0.0, 0.0, (0.0, 0.0), 1.0),
    (0.1, 1.0, 0.0, (0.0, 0.0), 1.0),
    (0.05, 0.3, 0.7, (0.0, 0.0), 2.0),
    (0.02, 0.4, 0.0, (0.6, 0.3), 1.0),
    (0.01, 0.2, 0.5, (0.7, 0.4), 0.5),
    (0.0, 0.0, 0.0, (1.0, 0.0), 1.0),
    (0.0, 0.0, 0.0, (0.0, 1.0), 1.0),
]
REG_BOUNDS = ["dct2", "dft", "zero", "dst1", ["dct1", "dst2", "replicate"]]
REG_SHAPES = {1: (13,), 2: (9, 8), 3: (7, 6, 5)}
REG_VS = [1.3, 0.8, 1.1]


def regulariser(S):
    """The reference's field and grid regularisers through its own wrappers
    (nitorch/_C/solve.py c_regulariser / c_regulariser_grid), float64, 1-3-D:
    every penalty mix of REG_FIELD / REG_GRID under every bound of
    REG_BOUNDS, weighted absolute / membrane, and each Hessian layout.
    Not generated, as the reference fails there: a call with every penalty
    zero (the field kernel's `zeros` never advances its channel loop), a 1-D
    field Hessian (the front-end expands it to 3-D), weighted field inputs
    with N > 1 (the kernel reads batch item 0's weights for every item) and
    grid Hessians with N > 1 (offset by the input's batch stride)."""
    import nitorch._C.solve as CS
    out = {}
    g = torch.Generator().manual_seed(123)
    for dim, shape in REG_SHAPES.items():
        vs = REG_VS[:dim]
        x = torch.randn((2, 2) + shape, generator=g, dtype=torch.float64)
        out[f"f{dim}_x"] = x.numpy()
        for kb, bnd in enumerate(REG_BOUNDS):
            bnd = bnd if isinstance(bnd, str) else bnd[:dim]
            for kp, (a, m, b, f) in enumerate(REG_FIELD):
                out[f"f{dim}_b{kb}_p{kp}"] = CS.c_regulariser(x, None, None, dim, a, m, b, f, vs, bnd).numpy()
        for kw, wc in enumerate((1, 2)):
            w = torch.rand((1, wc) + shape, generator=g, dtype=torch.float64) + 0.5
            out[f"f{dim}_w{kw}"] = w.numpy()
            for kp, (a, m) in enumerate((([0.2], [1.0, 0.5]), ([0.3], [0.0]))):
                out[f"f{dim}_w{kw}_p{kp}"] = CS.c_regulariser(x[:1], w, None, dim, a, m, [0.0], [1.0], vs,
                                                              "dct2").numpy()
        if dim > 1:
            x3 = torch.randn((2, 3) + shape, generator=g, dtype=torch.float64)
            out[f"f{dim}_x3"] = x3.numpy()
            for CC in (1, 3, 5, 6):
                h = torch.rand((2, CC) + shape, generator=g, dtype=torch.float64)
                out[f"f{dim}_h{CC}"] = h.numpy()
                out[f"f{dim}_h{CC}_out"] = CS.c_regulariser(x3, None, h, dim, [0.1], [0.5], [0.0], [1.0], vs,
                                                            "dft").numpy()
        v = torch.randn((2,) + shape + (dim,), generator=g, dtype=torch.float64)
        out[f"g{dim}_x"] = v.numpy()
        for kb, bnd in enumerate(REG_BOUNDS):
            bnd = bnd if isinstance(bnd, str) else bnd[:dim]
            for kp, (a, m, b, lame, f) in enumerate(REG_GRID):
                out[f"g{dim}_b{kb}_p{kp}"] = CS.c_regulariser_grid(v, None, None, a, m, b, lame, f, vs, bnd).numpy()
        w = torch.rand((2,) + shape, generator=g, dtype=torch.float64) + 0.5
        out[f"g{dim}_w"] = w.numpy()
        for kp, (a, m) in enumerate(((0.2, 1.0), (0.3, 0.0))):
            out[f"g{dim}_w_p{kp}"] = CS.c_regulariser_grid(v, w, None, a, m, 0.0, 0.0, 1.0, vs, "dft").numpy()
        if dim > 1:
            for DD in sorted({1, dim, dim * (dim + 1) // 2}):
                h = torch.rand((1,) + shape + (DD,), generator=g, dtype=torch.float64)
                out[f"g{dim}_h{DD}"] = h.numpy()
                out[f"g{dim}_h{DD}_out"] = CS.c_regulariser_grid(v[:1], None, h, 0.1, 0.5, 0.0, 0.0, 1.0, vs,
                                                                 "dct2").numpy()
    return {k: np.asarray(v) for k, v in out.items()}


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "regulariser":
        S = R.load_spatial()
        if S is None:
            raise SystemExit("reference tree / compiled backend not found")
        torch.set_num_threads(1)
        np.savez_compressed(os.path.join(HERE, "regulariser_golden.npz"), **regulariser(S))
        print("regulariser_golden.npz", os.path.getsize(os.path.join(HERE, "regulariser_golden.npz")))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "multires":
        S = R.load_spatial()
        ref = R.load_compiled()
        if S is None or ref is None:
            raise SystemExit("reference tree / compiled backend not found")
        torch.set_num_threads(1)
        np.savez_compressed(os.path.join(HERE, "multires_golden.npz"), **multires(ref, S))
        print("multires_golden.npz", os.path.getsize(os.path.join(HERE, "multires_golden.npz")))
        return
    if len(sys.argv) > 1 and sys.argv[1] == "spatial":
        S = R.load_spatial()
        if S is None:
            raise SystemExit("reference tree / compiled backend not found")
        torch.set_num_threads(1)
        np.savez_compressed(os.path.join(HERE, "spatial_golden.npz"), **spatial(S))
        print("spatial_golden.npz", os.path.getsize(os.path.join(HERE, "spatial_golden.npz")))
        return
    ref = R.load_compiled()
    if ref is None:
        raise SystemExit("build the reference first: python oracle/build_ref.py")
    torch.set_num_threads(1)
    np.savez_compressed(os.path.join(HERE, "pushpull_golden.npz"), **pushpull(ref))
    ts = R.load_ts_coeff()
    if ts is None:
        raise SystemExit("reference tree not found (NITORCH_REFERENCE)")
    np.savez_compressed(os.path.join(HERE, "coeff_golden.npz"), **coeff(ts))
    np.savez_compressed(os.path.join(HERE, "config1_golden.npz"), **config1(ref))
    for f in ("pushpull_golden.npz", "coeff_golden.npz", "config1_golden.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
