"""Python front-end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  The product (``nitorch_b200``) never does.

It wraps ``pushpull_oracle.c`` (a plain-C restatement of the reference's
push/pull and prefilter arithmetic, compiled by ``oracle/Makefile``) with
numpy-based functions that mirror the reference's native front-end
(``nitorch/_C/src/pushpull.cpp:76-327``): same argument meaning, same
output shapes, same mode wiring (``pushpull.cpp`` flag table).

Bounds and orders are given as lists of compiled-backend codes
(``nitorch/_C/src/bounds.h``: replicate 0, dct1 1, dct2 2, dst1 3, dst2 4,
dft 5, zero 7; orders 0-7), padded with the last entry as the reference's
allocator does (``pushpull_common.cpp:91-120``).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

PULL, PUSH, COUNT, GRAD, SGRAD = 1, 2, 4, 8, 16
QUIRK_D1, QUIRK_D3 = 1, 4

_LIBS = {}


def build():
    """Compile the oracle libraries (gcc only; seconds)."""
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib(real="f64"):
    if real not in _LIBS:
        path = os.path.join(BUILD, f"liboracle_{real}.so")
        if not os.path.exists(path):
            build()
        _LIBS[real] = _declare(ctypes.CDLL(path), real)
    return _LIBS[real]


def _ctype(real):
    return ctypes.c_double if real == "f64" else ctypes.c_float


def _declare(L, real):
    R = _ctype(real)
    i64 = ctypes.c_int64
    P = ctypes.c_void_p

    class Params(ctypes.Structure):
        _fields_ = [
            ("dim", ctypes.c_int), ("bound", ctypes.c_int * 3),
            ("order", ctypes.c_int * 3), ("extrapolate", ctypes.c_int),
            ("mode", ctypes.c_int), ("quirks", ctypes.c_int),
            ("N", i64), ("C", i64), ("src_size", i64 * 3),
            ("trgt_size", i64 * 3), ("trgt_K", i64),
            ("src", P), ("src_s", i64 * 5),
            ("trgt", P), ("trgt_s", i64 * 6),
            ("grid", P), ("grid_s", i64 * 5),
            ("out", P), ("out_s", i64 * 6),
            ("ggrad", P), ("ggrad_s", i64 * 5),
        ]

    L.Params = Params
    assert ctypes.sizeof(Params) == L.or_params_size(), "oracle ABI mismatch"
    L.or_pushpull.argtypes = [ctypes.POINTER(Params)]
    L.or_pushpull.restype = ctypes.c_int
    L.or_bound_index.argtypes = [ctypes.c_int, i64, i64]
    L.or_bound_index.restype = i64
    L.or_bound_sign.argtypes = [ctypes.c_int, i64, i64]
    L.or_bound_sign.restype = ctypes.c_int
    for name in ("or_weight", "or_fastweight", "or_fastgrad"):
        getattr(L, name).argtypes = [ctypes.c_int, R]
        getattr(L, name).restype = R
    L.or_fasthess.argtypes = [ctypes.c_int, R, ctypes.c_int]
    L.or_fasthess.restype = R
    L.or_support_low.argtypes = [ctypes.c_int, R]
    L.or_support_low.restype = i64
    L.or_coeff_axis.argtypes = [P, ctypes.c_int, ctypes.POINTER(i64),
                                ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.or_coeff_axis.restype = ctypes.c_int
    return L


def _pad(v, n):
    v = list(v) if isinstance(v, (list, tuple)) else [v]
    v = v + v[-1:] * max(0, n - len(v))
    return [int(x) for x in v[:n]] + [0] * (3 - n)


def _strides(a):
    return [s // a.itemsize for s in a.strides]


def _np(real):
    return np.float64 if real == "f64" else np.float32


def _run(real, dim, bound, order, extrapolate, mode, *, src=None, src_size,
         trgt=None, grid, out=None, ggrad=None, trgt_K=0, quirks=0):
    L = lib(real)
    p = L.Params()
    p.dim = dim
    p.bound[:] = _pad(bound, dim)
    p.order[:] = _pad(order, dim)
    p.extrapolate = int(extrapolate)
    p.mode = mode
    p.quirks = quirks
    p.N = grid.shape[0]
    p.C = (src.shape[1] if src is not None else
           trgt.shape[1] if trgt is not None else 1)
    p.src_size[:] = list(src_size) + [1] * (3 - dim)
    p.trgt_size[:] = list(grid.shape[1:1 + dim]) + [1] * (3 - dim)
    p.trgt_K = trgt_K

    def put(name, arr, nstride):
        if arr is None:
            setattr(p, name, None)
            return
        s = _strides(arr)
        full = [0] * nstride
        setattr(p, name, arr.ctypes.data)
        return s, full

    if src is not None:
        s = _strides(src)
        p.src = src.ctypes.data
        p.src_s[:] = s[:2] + s[2:2 + dim] + [0] * (3 - dim)
    if trgt is not None:
        s = _strides(trgt)
        p.trgt = trgt.ctypes.data
        sk = s[2 + dim] if trgt.ndim == dim + 3 else 0
        p.trgt_s[:] = s[:2] + s[2:2 + dim] + [0] * (3 - dim) + [sk]
    s = _strides(grid)
    p.grid = grid.ctypes.data
    p.grid_s[:] = [s[0]] + s[1:1 + dim] + [0] * (3 - dim) + [s[1 + dim]]
    if out is not None:
        s = _strides(out)
        p.out = out.ctypes.data
        sk = s[2 + dim] if out.ndim == dim + 3 else 0
        p.out_s[:] = s[:2] + s[2:2 + dim] + [0] * (3 - dim) + [sk]
    if ggrad is not None:
        s = _strides(ggrad)
        p.ggrad = ggrad.ctypes.data
        p.ggrad_s[:] = [s[0]] + s[1:1 + dim] + [0] * (3 - dim) + [s[1 + dim]]
    rc = L.or_pushpull(ctypes.byref(p))
    if rc != 0:
        raise RuntimeError(f"oracle failed with {rc}")


def _prep(real, *arrays):
    dt = _np(real)
    return [None if a is None else np.asarray(a, dtype=dt) for a in arrays]


# --------------------------------------------------------------------- #
# The eight reference operations (pushpull.cpp:76-327)                  #
# --------------------------------------------------------------------- #

def grid_pull(inp, grid, bound, order, extrapolate, real="f64", quirks=0):
    inp, grid = _prep(real, inp, grid)
    dim = grid.shape[-1]
    out = np.zeros(inp.shape[:2] + grid.shape[1:1 + dim], dtype=inp.dtype)
    _run(real, dim, bound, order, extrapolate, PULL, src=inp,
         src_size=inp.shape[2:], grid=grid, out=out, quirks=quirks)
    return out


def grid_pull_backward(grad, inp, grid, bound, order, extrapolate,
                       need_input=True, need_grid=True, real="f64", quirks=0):
    grad, inp, grid = _prep(real, grad, inp, grid)
    dim = grid.shape[-1]
    res = []
    gi = np.zeros(inp.shape, inp.dtype) if need_input else None
    gg = np.zeros(grid.shape, grid.dtype) if need_grid else None
    mode = (PUSH if need_input else 0) | (GRAD if need_grid else 0)
    if mode:
        _run(real, dim, bound, order, extrapolate, mode, src=inp,
             src_size=inp.shape[2:], trgt=grad, grid=grid, out=gi, ggrad=gg,
             quirks=quirks)
    if need_input:
        res.append(gi)
    if need_grid:
        res.append(gg)
    return res


def grid_push(inp, grid, shape, bound, order, extrapolate, real="f64", quirks=0):
    inp, grid = _prep(real, inp, grid)
    dim = grid.shape[-1]
    shape = tuple(shape) if shape else tuple(inp.shape[2:])
    out = np.zeros(inp.shape[:2] + shape, dtype=inp.dtype)
    _run(real, dim, bound, order, extrapolate, PUSH, src_size=shape,
         trgt=inp, grid=grid, out=out, quirks=quirks)
    return out


def grid_push_backward(grad, inp, grid, bound, order, extrapolate,
                       need_input=True, need_grid=True, real="f64", quirks=0):
    grad, inp, grid = _prep(real, grad, inp, grid)
    dim = grid.shape[-1]
    res = []
    gi = np.zeros(inp.shape, inp.dtype) if need_input else None
    gg = np.zeros(grid.shape, grid.dtype) if need_grid else None
    mode = (PULL if need_input else 0) | (GRAD if need_grid else 0)
    if mode:
        _run(real, dim, bound, order, extrapolate, mode, src=grad,
             src_size=grad.shape[2:], trgt=inp, grid=grid, out=gi, ggrad=gg,
             quirks=quirks)
    if need_input:
        res.append(gi)
    if need_grid:
        res.append(gg)
    return res


def grid_count(grid, shape, bound, order, extrapolate, real="f64", quirks=0):
    (grid,) = _prep(real, grid)
    dim = grid.shape[-1]
    shape = tuple(shape) if shape else tuple(grid.shape[1:1 + dim])
    out = np.zeros((grid.shape[0], 1) + shape, dtype=grid.dtype)
    _run(real, dim, bound, order, extrapolate, COUNT, src_size=shape,
         grid=grid, out=out, quirks=quirks)
    return out


def grid_count_backward(grad, grid, bound, order, extrapolate, real="f64",
                        quirks=0):
    grad, grid = _prep(real, grad, grid)
    dim = grid.shape[-1]
    gg = np.zeros(grid.shape, grid.dtype)
    _run(real, dim, bound, order, extrapolate, GRAD, src=grad,
         src_size=grad.shape[2:], grid=grid, ggrad=gg, quirks=quirks)
    return gg


def grid_grad(inp, grid, bound, order, extrapolate, real="f64", quirks=0):
    inp, grid = _prep(real, inp, grid)
    dim = grid.shape[-1]
    out = np.zeros(inp.shape[:2] + grid.shape[1:1 + dim] + (dim,), inp.dtype)
    _run(real, dim, bound, order, extrapolate, SGRAD, src=inp,
         src_size=inp.shape[2:], grid=grid, out=out, quirks=quirks)
    return out


def grid_grad_backward(grad, inp, grid, bound, order, extrapolate,
                       need_input=True, need_grid=True, real="f64", quirks=0):
    grad, inp, grid = _prep(real, grad, inp, grid)
    dim = grid.shape[-1]
    res = []
    gi = np.zeros(inp.shape, inp.dtype) if need_input else None
    gg = np.zeros(grid.shape, grid.dtype) if need_grid else None
    mode = (PUSH if need_input else 0) | (GRAD if need_grid else 0)
    if mode:
        _run(real, dim, bound, order, extrapolate, mode, src=inp,
             src_size=inp.shape[2:], trgt=grad, grid=grid, out=gi, ggrad=gg,
             trgt_K=dim, quirks=quirks)
    if need_input:
        res.append(gi)
    if need_grid:
        res.append(gg)
    return res


# --------------------------------------------------------------------- #
# Prefilter (_ts/coeff.py:285-344), FP64                                #
# --------------------------------------------------------------------- #

def spline_coeff(inp, bound_ts, order, dim=-1):
    """One axis.  ``bound_ts`` uses the prefilter's integer codes
    (_ts/bounds.py:7-14): zero 0, replicate 1, dct1 2, dct2 3, dft 6."""
    a = np.ascontiguousarray(np.asarray(inp, dtype=np.float64)).copy()
    axis = dim % a.ndim
    shape = (ctypes.c_int64 * a.ndim)(*a.shape)
    rc = lib("f64").or_coeff_axis(a.ctypes.data, a.ndim, shape, axis,
                                  int(bound_ts), int(order))
    if rc == -2:
        raise NotImplementedError("prefilter bound not implemented")
    if rc:
        raise ValueError(f"prefilter failed with {rc}")
    return a


def spline_coeff_nd(inp, bound_ts, order, dim=None):
    a = np.asarray(inp, dtype=np.float64)
    dim = a.ndim if dim is None else dim
    b = _pad(bound_ts, dim)[:dim]
    o = _pad(order, dim)[:dim]
    for d in range(dim):
        a = spline_coeff(a, b[d], o[d], dim=-dim + d)
    return a


# compiled-backend bound code -> prefilter code (grid.py:133 via _TSBoundType)
BOUND_TO_TS = {0: 1, 1: 2, 2: 3, 3: 4, 4: 5, 5: 6, 7: 0}


# --------------------------------------------------------------------- #
# Stationary velocity fields: scaling and squaring (FP64)               #
# --------------------------------------------------------------------- #

def _identity_np(shape):
    mesh = np.meshgrid(*[np.arange(s, dtype=np.float64) for s in shape], indexing="ij")
    return np.stack(mesh, -1)


def svf_compose(u, bound=5, order=1, extrapolate=1):
    """u + pull(u, id + u) for a displacement u (N, *spatial, D): the step of
    nitorch/spatial/_svf.py:85-94, with _pull_vel (:323-362) moving the
    components to the channel axis and pulling at id + u."""
    u = np.asarray(u, np.float64)
    img = np.moveaxis(u, -1, 1)
    grid = _identity_np(u.shape[1:-1])[None] + u
    pulled = grid_pull(img, grid, [bound], [order], extrapolate)
    return u + np.moveaxis(pulled, 1, -1)


def svf_compose_backward(g, u, bound=5, order=1, extrapolate=1):
    """Exact gradient of <g, svf_compose(u)> w.r.t. u: g, plus the pull's
    input gradient (a push of g) and its grid gradient (d grid / d u = I)."""
    u = np.asarray(u, np.float64)
    g = np.asarray(g, np.float64)
    img = np.moveaxis(u, -1, 1)
    grid = _identity_np(u.shape[1:-1])[None] + u
    gi, gg = grid_pull_backward(np.moveaxis(g, -1, 1), img, grid, [bound], [order], extrapolate)
    return g + np.moveaxis(gi, 1, -1) + gg


def svf_exp(vel, steps=8, bound=5, order=1, inverse=False, displacement=False):
    """nitorch/spatial/_svf.py:47-98 (exp_forward): scale by 2^-steps, then
    `steps` self-compositions; returns the transformation (id + u) unless
    `displacement`.  vel: (N, *spatial, D)."""
    u = (-1.0 if inverse else 1.0) * np.asarray(vel, np.float64) / 2 ** steps
    for _ in range(steps):
        u = svf_compose(u, bound, order)
    return u if displacement else u + _identity_np(u.shape[1:-1])[None]


def svf_exp_backward(vel, grad, steps=8, bound=5, order=1, inverse=False):
    """Gradient of <grad, svf_exp(vel)> w.r.t. vel by the chain rule through
    the compositions (what autograd computes on the reference's default
    path)."""
    u = (-1.0 if inverse else 1.0) * np.asarray(vel, np.float64) / 2 ** steps
    states = []
    for _ in range(steps):
        states.append(u)
        u = svf_compose(u, bound, order)
    g = np.asarray(grad, np.float64)
    for s in reversed(states):
        g = svf_compose_backward(g, s, bound, order)
    return (-1.0 if inverse else 1.0) * g / 2 ** steps


# --------------------------------------------------------------------- #
# Jacobians of transformation fields (FP64)                             #
# --------------------------------------------------------------------- #

def _central_diff1d(x, axis, bound, vs):
    """nitorch/spatial/_finite_differences.py:32-222, order 1, side 'c':
    (x[i+1] - x[i-1]) / (2 vs) with the bound's value beyond each end; a
    singleton axis returns x itself (:87-91)."""
    x = np.moveaxis(np.asarray(x, np.float64), axis, 0)
    n = x.shape[0]
    if n == 1:
        return np.moveaxis(x.copy(), 0, axis)
    d = np.empty_like(x)
    d[1:-1] = x[2:] - x[:-2]
    if bound in ("dct2", "replicate"):
        d[0] = x[1] - x[0]
        d[-1] = x[-1] - x[-2]
    elif bound == "dct1":
        d[0] = 0
        d[-1] = 0
    elif bound == "dst2":
        d[0] = x[1] + x[0]
        d[-1] = -(x[-1] + x[-2])
    elif bound in ("dst1", "zero"):
        d[0] = x[1]
        d[-1] = -x[-2]
    elif bound == "dft":
        d[0] = x[1] - x[-1]
        d[-1] = x[0] - x[-2]
    else:
        raise ValueError(bound)
    d /= 2 * vs
    return np.moveaxis(d, 0, axis)


def grid_jacobian(grid, bound="dft", voxel_size=1, type="grid", add_identity=True):
    """nitorch/spatial/_grid.py:917-969 without `sample`: central finite
    differences of the displacement; jac[..., i, j] = d psi_i / d x_j.
    grid: (N, *spatial, D)."""
    g = np.asarray(grid, np.float64)
    D = g.shape[-1]
    spatial = g.shape[1:-1]
    vs = list(voxel_size) if isinstance(voxel_size, (list, tuple)) else [voxel_size] * D
    if type == "grid":
        g = g - _identity_np(spatial)[None]
    jac = np.stack([_central_diff1d(g, 1 + j, bound, vs[j]) for j in range(D)], -1)
    if add_identity:
        for i in range(D):
            jac[..., i, i] += 1
    return jac


def grid_jacdet(grid, bound="dft", voxel_size=1, type="grid", add_identity=True):
    """nitorch/spatial/_grid.py:972-1013: det of grid_jacobian."""
    return np.linalg.det(grid_jacobian(grid, bound, voxel_size, type, add_identity))


# ---------------------------------------------------------------------------
# Multigrid prolongation / restriction and nitorch's native resize
# ---------------------------------------------------------------------------

def _bound_index(b, i, n):
    """Node i of an n-voxel axis under bound code b (nitorch/_C/src/
    bounds_common.h:26-120: replicate clamps; dct1 reflects about the end
    centres, period 2(n-1); dct2 / dst2 about the end edges, period 2n;
    dst1 antisymmetric about the centres, period 2(n+1); dft wraps)."""
    if b == 0:
        return min(max(i, 0), n - 1)
    if b == 1:
        if n == 1:
            return 0
        p = 2 * (n - 1)
        i = abs(i) % p
        return p - i if i >= n else i
    if b in (2, 4):
        p = 2 * n
        i = (p - ((-i - 1) % p) - 1) if i < 0 else i % p
        return p - i - 1 if i >= n else i
    if b == 3:
        if n == 1:
            return 0
        p = 2 * (n + 1)
        i = 0 if i == -1 else (-i - 2 if i < 0 else i)
        i %= p
        return n - 1 if i == n else (p - i - 2 if i > n else i)
    if b == 5:
        return i % n
    return i


def _bound_sign(b, i, n):
    """Sign of node i under bound code b (bounds_common.h:122-160): dst1 is
    zero on its mirror nodes and alternates between periods, dst2
    alternates, zero is 0 outside the axis."""
    if b == 3:
        if n == 1:
            return 1
        p = 2 * (n + 1)
        i = n - i - 1 if i < 0 else i
        i %= p
        if i % (n + 1) == n:
            return 0
        return -1 if (i // (n + 1)) % 2 else 1
    if b == 4:
        i = n - i - 1 if i < 0 else i
        return -1 if (i // n) % 2 else 1
    if b == 7:
        return 0 if (i < 0 or i >= n) else 1
    return 1


def _quadratic(d):
    """Quadratic B-spline (interpolation_common.h, order 2)."""
    d = abs(d)
    if d < 0.5:
        return 0.75 - d * d
    if d < 1.5:
        return 0.5 * (1.5 - d) ** 2
    return 0.0


def _multires_matrix(n_in, n_out, b, restrict):
    """(n_out, n_in) matrix of one axis of fmg_prolongation / fmg_restriction
    (nitorch/_C/src/impl/multires_common.cpp:419-500 and 587-660): output
    voxel o reads x = (o + 1/2) s - 1/2, s = n_in / n_out.  Prolongation:
    nodes floor(x + 1/2) - 1 .. + 1, quadratic B-spline weights.
    Restriction: nodes floor(x) - 1 .. + 2, weight L(|x - i| / s) / s with
    L the linear B-spline.  Boundary index and sign per node."""
    s = n_in / n_out
    M = np.zeros((n_out, n_in))
    for o in range(n_out):
        x = (o + 0.5) * s - 0.5
        if restrict:
            i1 = int(np.floor(x))
            nodes = [(i, max(0.0, 1.0 - abs(x - i) / s) / s) for i in range(i1 - 1, i1 + 3)]
        else:
            i1 = int(np.floor(x + 0.5))
            nodes = [(i, _quadratic(x - i)) for i in range(i1 - 1, i1 + 2)]
        for i, w in nodes:
            sg = _bound_sign(b, i, n_in)
            if sg:
                M[o, _bound_index(b, i, n_in)] += sg * w
    return M


def _apply_axes(x, mats):
    """Apply one matrix per spatial axis of x (N, C, *spatial)."""
    y = np.asarray(x, np.float64)
    for d, M in enumerate(mats):
        y = np.moveaxis(np.tensordot(M, np.moveaxis(y, 2 + d, 0), axes=(1, 0)), 0, 2 + d)
    return y


def fmg_prolongation(inp, bound=(2,), shape=None):
    """nitorch's native fmg_prolongation (nitorch/_C/src/multires.cpp:24-48):
    inp (N, C, *spatial) with 1-3 spatial axes; output shape floor(2 s) per
    axis unless `shape` is given."""
    sp = inp.shape[2:]
    shape = shape or [int(np.floor(2.0 * s)) for s in sp]
    b = _pad(list(bound), len(sp))
    return _apply_axes(inp, [_multires_matrix(sp[d], shape[d], b[d], False) for d in range(len(sp))])


def fmg_restriction(inp, bound=(2,), shape=None):
    """nitorch's native fmg_restriction (multires.cpp:50-74): output shape
    ceil(s / 2) per axis unless `shape` is given."""
    sp = inp.shape[2:]
    shape = shape or [int(np.ceil(s / 2.0)) for s in sp]
    b = _pad(list(bound), len(sp))
    return _apply_axes(inp, [_multires_matrix(sp[d], shape[d], b[d], True) for d in range(len(sp))])


def _padf(v, n):
    v = list(v) if isinstance(v, (list, tuple)) else [v]
    return [float(x) for x in (v + v[-1:] * max(0, n - len(v)))[:n]]


def resize_affine(factor, n_src, n_tgt, mode):
    """(shift, scale) of one axis of ni::resize (nitorch/_C/src/impl/
    resize_common.cpp:1547-1566): target voxel w reads source x = scale w +
    shift.  Modes: 0 edge, 1 center, 2 first, 3 last.  IEEE division, as
    there: a one-voxel axis gives inf / nan in the center and last modes."""
    f, ns, nt = np.float64(factor), np.float64(n_src), np.float64(n_tgt)
    with np.errstate(divide="ignore", invalid="ignore"):
        shift, scale = np.float64(0.0), 1.0 / f
        if mode == 0:
            shift, scale = 0.5 * (ns / nt - 1), ns / nt
        elif mode == 1:
            shift, scale = np.float64(0.0), (ns - 1) / (nt - 1)
        elif mode == 3:
            shift = f * (ns - 1) / (nt - 1)
    return float(shift), float(scale)


def resize_native(inp, out_shape=None, factor=(1.0,), bound=(2,), order=(1,), mode=(1,), adjoint=False,
                  normalize=False):
    """nitorch's native resize (nitorch/_C/src/resize.cpp:19-60,
    impl/resize_common.cpp:1488-1660) on inp (N, C, *spatial): the pull of
    the source at the target lattice's diagonal map, always extrapolating,
    or (adjoint) the push of the target into the source lattice, then the
    optional normalisation by the product of the scales.  The reference
    runs 3-D inputs only (1-D / 2-D ones raise an index error in its
    allocator); here the 1-D / 2-D normalisation is the product over the
    real axes."""
    D = inp.ndim - 2
    f = _padf(factor, 3)
    if adjoint:
        f = [1.0 / v for v in f]
    if adjoint:
        tgt_shape = list(inp.shape[2:])
        src_shape = list(out_shape) if out_shape else [int(np.ceil(s * f[d])) for d, s in enumerate(tgt_shape)]
    else:
        src_shape = list(inp.shape[2:])
        tgt_shape = list(out_shape) if out_shape else [int(np.floor(s * f[d])) for d, s in enumerate(src_shape)]
    m = _pad(list(mode), 3)
    m = m[:D] + [m[D - 1]] * (3 - D)
    full_src = src_shape + [1] * (3 - D)
    full_tgt = tgt_shape + [1] * (3 - D)
    aff = [resize_affine(f[d], float(full_src[d]), float(full_tgt[d]), m[d]) for d in range(3)]
    axes = [np.arange(tgt_shape[d], dtype=np.float64) * aff[d][1] + aff[d][0] for d in range(D)]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), -1)[None]
    grid = np.broadcast_to(grid, (inp.shape[0],) + grid.shape[1:]).copy()
    if adjoint:
        out = grid_push(inp, grid, src_shape, bound, order, 1)
    else:
        out = grid_pull(inp, grid, bound, order, 1)
    if normalize:
        out = out * float(np.prod([aff[d][1] for d in range(D)]))
    return out


def _edge_grid(src_shape, tgt_shape, N):
    """(N, *tgt, D) coordinates of the edge-aligned map of the multigrid
    solvers (nitorch/spatial/_solvers.py:170-177): arange(tgt) * src / tgt +
    0.5 (src / tgt - 1) per axis, in the input's dtype (float64 here)."""
    axes = [np.arange(t, dtype=np.float64) * (s / t) + 0.5 * (s / t - 1) for s, t in zip(src_shape, tgt_shape)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1)[None]
    return np.broadcast_to(g, (N,) + g.shape[1:]).copy()


def solver_prolong(x, shape=None, bound=2, order=2):
    """nitorch/spatial/_solvers.py:147-181: x (N, *spatial, K) pulled at the
    edge-aligned map of a `shape` lattice (default 2 * spatial), order 2,
    extrapolating."""
    sp = x.shape[1:-1]
    shape = list(shape) if shape else [2 * s for s in sp]
    grid = _edge_grid(sp, shape, x.shape[0])
    y = grid_pull(np.moveaxis(x, -1, 1), grid, [bound], [order], 1)
    return np.moveaxis(y, 1, -1)


def solver_restrict(x, shape=None, bound=2, order=1):
    """nitorch/spatial/_solvers.py:184-224: x (N, *spatial, K) pushed from
    the edge-aligned map onto a `shape` lattice (default ceil(spatial / 2)),
    order 1, extrapolating, times prod(shape) / prod(spatial)."""
    sp = x.shape[1:-1]
    shape = list(shape) if shape else [int(np.ceil(s / 2)) for s in sp]
    grid = _edge_grid(shape, sp, x.shape[0])
    y = grid_push(np.moveaxis(x, -1, 1), grid, shape, [bound], [order], 1)
    return np.moveaxis(y, 1, -1) * (np.prod(shape) / np.prod(sp))


# ---------------------------------------------------------------------------
# Field and grid regularisers (nitorch._C.solve.c_regulariser /
# c_regulariser_grid; kernels nitorch/_C/src/impl/regulariser_common.cpp and
# regulariser_grid_common.cpp).  Every mode of the reference is a linear
# stencil: differences to the centre along +-1 and +-2 steps of an axis and
# along the diagonals of an axis pair, plus (grids) the Lame cross terms and
# (both) the Hessian product at the voxel.  Neighbours are read with the
# boundary index and sign of every axis they step along; a difference is
# sign * value(neighbour) - value(centre), as the reference forms it.
# ---------------------------------------------------------------------------

def _unfold3(v, default):
    """VEC_UNFOLD (regulariser_common.cpp:30-36): three entries, the last
    given one repeated, `default` when empty."""
    v = [float(x) for x in v] if v is not None else []
    if not v:
        return [default] * 3
    return [v[min(i, len(v) - 1)] for i in range(3)]


def _per_channel(v, C):
    """set_factors (regulariser_common.cpp:263-280): C entries, the last given
    one repeated, 0 when empty."""
    v = [float(x) for x in v] if v is not None else []
    if not v:
        return [0.0] * C
    return [v[min(c, len(v) - 1)] for c in range(C)]


class _Nbr:
    """Neighbour gather for the regularisers: value(x + o) of an (N, K,
    *spatial) array for an offset vector o, with boundary index and sign."""

    def __init__(self, shape, bounds):
        self.shape = shape
        self.bounds = bounds
        self.cache = {}

    def axis(self, a, o):
        key = (a, o)
        if key not in self.cache:
            n = self.shape[a]
            # zero bound: out-of-axis nodes carry sign 0 (index clipped for the read)
            idx = np.array([min(max(_bound_index(self.bounds[a], i + o, n), 0), n - 1) for i in range(n)])
            sgn = np.array([_bound_sign(self.bounds[a], i + o, n) for i in range(n)], dtype=np.float64)
            self.cache[key] = (idx, sgn)
        return self.cache[key]

    def get(self, arr, offs):
        """sign * arr at the offset neighbour of every voxel (arr: (..., *spatial))."""
        dim = len(self.shape)
        out = arr
        sign = np.ones(self.shape)
        for a in range(dim):
            if offs[a] == 0:
                continue
            idx, sgn = self.axis(a, offs[a])
            out = np.take(out, idx, axis=arr.ndim - dim + a)
            shp = [1] * dim
            shp[a] = self.shape[a]
            sign = sign * sgn.reshape(shp)
        return out * sign


def _step(dim, a, s):
    o = [0] * dim
    o[a] = s
    return o


def _diag(dim, a, b, sa, sb):
    o = [0] * dim
    o[a] = sa
    o[b] = sb
    return o


def _hessian_field(h, u, C):
    """matvec_eye / _diag / _estatics / _sym (regulariser_common.cpp:592-672)
    of an (N, CC, *spatial) Hessian and an (N, C, *spatial) field."""
    CC = h.shape[1]
    out = np.zeros_like(u)
    if CC == 1:
        return h[:, :1] * u
    if CC == C:
        return h * u
    if CC == 2 * C - 1:
        r = h[:, C - 1]
        s = u[:, C - 1]
        acc = s * r
        for c in range(C - 1):
            out[:, c] += h[:, c] * u[:, c] + h[:, C + c] * s
            acc = acc + h[:, C + c] * u[:, c]
        out[:, C - 1] += acc
        return out
    k = C
    for c in range(C):
        out[:, c] += h[:, c] * u[:, c]
    for c in range(C):
        for cc in range(c + 1, C):
            out[:, cc] += h[:, k] * u[:, c]
            out[:, c] += h[:, k] * u[:, cc]
            k += 1
    return out


def regulariser(x, weight=None, hessian=None, absolute=(), membrane=(), bending=(), voxel_size=(1.0,),
                bound=(2,)):
    """(H + L) x for an (N, C, *spatial) field, 1-3-D
    (regulariser_common.cpp: set_kernel :285-299, vel2mom3d_bending :752-804,
    _membrane :808-839, _absolute :843-856, _rls_membrane :860-903,
    _rls_absolute :907-925, and their 2-D / 1-D forms).  weight (N, C|1,
    *spatial) weights the absolute and membrane energies (bending with a
    weight is an error, as there); hessian (N, CC, *spatial), CC in {1, C,
    2C-1, C(C+1)/2}.  Weights are read per batch item."""
    x = np.asarray(x, np.float64)
    N, C = x.shape[:2]
    shape = x.shape[2:]
    dim = len(shape)
    a = _per_channel(absolute, C)
    m = _per_channel(membrane, C)
    b = _per_channel(bending, C)
    vs = _unfold3(voxel_size, 1.0)
    vx = [1.0 / (v * v) for v in vs]
    vx = [vx[i] if i < dim else 0.0 for i in range(3)]
    bnd = [int(v) for v in _unfold3(bound, 0.0)]
    nb = _Nbr(shape, bnd)
    svx = sum(vx)
    m1 = [-vx[i] for i in range(3)]
    b1 = [-4.0 * vx[i] * svx for i in range(3)]
    b2 = [vx[i] * vx[i] for i in range(3)]
    out = np.zeros_like(x)
    w = None
    if weight is not None:
        if any(b):
            raise ValueError("RLS only implemented for absolute/membrane")
        w = np.broadcast_to(np.asarray(weight, np.float64), x.shape)
    for c in range(C):
        u = x[:, c]
        if w is not None:
            wc = w[:, c]
            acc = a[c] * wc * u
            if m[c]:
                sm = np.zeros_like(u)
                for ax in range(dim):
                    for s in (-1, 1):
                        o = _step(dim, ax, s)
                        sm += m1[ax] * (wc + nb.get(wc, o)) * (nb.get(u, o) - u)
                acc = acc + m[c] * 0.5 * sm
            out[:, c] = acc
            continue
        acc = a[c] * u
        for ax in range(dim):
            w1 = m[c] * m1[ax] + b[c] * b1[ax]
            acc = acc + w1 * (nb.get(u, _step(dim, ax, -1)) - u + nb.get(u, _step(dim, ax, 1)) - u)
        if b[c]:
            bb = np.zeros_like(u)
            for ax in range(dim):
                bb += b2[ax] * (nb.get(u, _step(dim, ax, -2)) - u + nb.get(u, _step(dim, ax, 2)) - u)
            for i in range(dim):
                for j in range(i + 1, dim):
                    wp = 2.0 * vx[i] * vx[j]
                    for si in (-1, 1):
                        for sj in (-1, 1):
                            bb += wp * (nb.get(u, _diag(dim, i, j, si, sj)) - u)
            acc = acc + b[c] * bb
        out[:, c] = acc
    if hessian is not None:
        h = np.broadcast_to(np.asarray(hessian, np.float64), (N, np.asarray(hessian).shape[1]) + shape)
        out = out + _hessian_field(h, x, C)
    return out


def regulariser_grid(x, weight=None, hessian=None, absolute=0.0, membrane=0.0, bending=0.0, shear=0.0, div=0.0,
                     voxel_size=(1.0,), bound=(5,)):
    """(H + L) x for an (N, D, *spatial) displacement field (components
    second, as the native front-end takes it), 1-3-D
    (regulariser_grid_common.cpp: set_kernel :265-298; vel2mom3d_lame
    :927-1084, _all, _bending, _membrane :1088-1144, _absolute :1147-1166,
    _rls_membrane, _rls_absolute, and their 2-D / 1-D forms).  Component d
    is scaled by the squared voxel size of its axis; the Lame terms (shear
    mu, divergence lambda) couple the components.  weight (N, *spatial)
    weights absolute and membrane (an error with bending or Lame, as
    there); hessian (N, DD, *spatial), DD in {1, D, D(D+1)/2}."""
    x = np.asarray(x, np.float64)
    N, D = x.shape[:2]
    shape = x.shape[2:]
    dim = len(shape)
    vs = _unfold3(voxel_size, 1.0)
    vx = [1.0 / (v * v) for v in vs]
    vx = [vx[i] if i < dim else 0.0 for i in range(3)]
    bnd = [int(v) for v in _unfold3(bound, 0.0)]
    nb = _Nbr(shape, bnd)
    lam0, lam1, lam2, mu, lam = float(absolute), float(membrane), float(bending), float(shear), float(div)
    svx = sum(vx)
    w1 = [lam2 * (-4.0 * vx[i] * svx) - lam1 * vx[i] for i in range(3)]
    w2 = [lam2 * vx[i] * vx[i] for i in range(3)]
    wc2 = 0.25 * mu + 0.25 * lam
    out = np.zeros_like(x)
    if weight is not None:
        if lam2 or mu or lam:
            raise ValueError("RLS only implemented for absolute/membrane")
        wg = np.broadcast_to(np.asarray(weight, np.float64).reshape((-1,) + shape), (N,) + shape)
        for d in range(D):
            u = x[:, d]
            acc = lam0 * wg * u
            if lam1:
                sm = np.zeros_like(u)
                for ax in range(dim):
                    for s in (-1, 1):
                        o = _step(dim, ax, s)
                        sm += w1[ax] * (wg + nb.get(wg, o)) * (nb.get(u, o) - u)
                acc = acc + sm * 0.5
            out[:, d] = acc / vx[d]
    else:
        for d in range(D):
            u = x[:, d]
            acc = lam0 * u
            for ax in range(dim):
                acc = acc + w1[ax] * (nb.get(u, _step(dim, ax, -1)) - u + nb.get(u, _step(dim, ax, 1)) - u)
            if lam2:
                for ax in range(dim):
                    acc = acc + w2[ax] * (nb.get(u, _step(dim, ax, -2)) - u + nb.get(u, _step(dim, ax, 2)) - u)
                for i in range(dim):
                    for j in range(i + 1, dim):
                        wp = lam2 * 2.0 * vx[i] * vx[j]
                        for si in (-1, 1):
                            for sj in (-1, 1):
                                acc = acc + wp * (nb.get(u, _diag(dim, i, j, si, sj)) - u)
            res = acc / vx[d]
            if mu or lam:
                for ax in range(dim):
                    lw = (-2.0 * mu - lam) if ax == d else (-mu * vx[ax] / vx[d])
                    res = res + lw * (nb.get(u, _step(dim, ax, -1)) - u + nb.get(u, _step(dim, ax, 1)) - u)
                for e in range(D):
                    if e == d:
                        continue
                    for sd in (-1, 1):
                        for se in (-1, 1):
                            res = res - wc2 * sd * se * nb.get(x[:, e], _diag(dim, d, e, sd, se))
            out[:, d] = res
    if hessian is not None:
        h = np.asarray(hessian, np.float64)
        h = np.broadcast_to(h, (N, h.shape[1]) + shape)
        DD = h.shape[1]
        if DD == 1:
            out = out + h[:, :1] * x
        elif DD == D:
            out = out + h * x
        else:
            k = D
            hx = h[:, :D] * x
            for i in range(D):
                for j in range(i + 1, D):
                    hx[:, i] += h[:, k] * x[:, j]
                    hx[:, j] += h[:, k] * x[:, i]
                    k += 1
            out = out + hx
    return out
