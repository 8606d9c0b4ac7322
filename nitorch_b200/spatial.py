"""Drop-in replacement for nitorch's compiled backend module ``nitorch._C.spatial``.

Exposes the eight push/pull functions and the two enums with the signatures
of ``nitorch/_C/spatial.cpp:82-89`` (C++: ``nitorch/_C/src/pushpull.h:10-57``):

    grid_pull(input, grid, bound, interpolation, extrapolate) -> Tensor
    grid_pull_backward(grad, input, grid, bound, interpolation, extrapolate) -> list
    grid_push(input, grid, shape, bound, interpolation, extrapolate) -> Tensor
    grid_push_backward(grad, input, grid, bound, interpolation, extrapolate) -> list
    grid_count(grid, shape, bound, interpolation, extrapolate) -> Tensor
    grid_count_backward(grad, grid, bound, interpolation, extrapolate) -> Tensor
    grid_grad(input, grid, bound, interpolation, extrapolate) -> Tensor
    grid_grad_backward(grad, input, grid, bound, interpolation, extrapolate) -> list

and the native multigrid resampling the same module binds
(``nitorch/_C/spatial.cpp:101-110``; defined in ``nitorch_b200.multires``):

    resize(input, output, factor, bound, interpolation, mode, do_adjoint, normalize)
    resize_backward / prolongation / prolongation_backward / restriction /
    restriction_backward / fmg_prolongation(input, output, bound) / fmg_restriction
    and the enum GridAlignType

``bound`` / ``interpolation`` are lists (one entry per axis, padded with the
last one); ``extrapolate`` is an int bit field.  As in the reference, the
backward functions read ``requires_grad`` of ``input`` / ``grid`` to decide
which gradients to compute, and return them in that order
(``nitorch/_C/src/pushpull.cpp:110-125,188-203,256-272,310-325``).

Argument errors raise ``RuntimeError`` with the reference's "(): expected
..." wording (``pushpull.cpp:19-72``).  Differences, by design:
  * CUDA tensors only -- there is no CPU path (the call raises);
  * bfloat16 / float16 images may be paired with a float32 grid (images are
    stored in 16 bits, all arithmetic is float32);
  * per-axis orders are honoured on every axis (the reference uses the
    second axis' order for the third, ``pushpull_common.cpp:591``).
"""
import ctypes
import os
import threading
import weakref

import torch

from . import _lib
from .enums import BoundType, InterpolationType

__all__ = ["grid_pull", "grid_pull_backward", "grid_push", "grid_push_backward",
           "grid_count", "grid_count_backward", "grid_grad", "grid_grad_backward",
           "BoundType", "InterpolationType", "set_deterministic", "get_deterministic",
           "set_sample_order", "sample_order", "grid_pull_push", "grid_pull_push_backward"]

_FLOATS = (torch.float32, torch.float64, torch.bfloat16, torch.float16)
_deterministic = bool(int(os.environ.get("PP_DETERMINISTIC", "0") or "0"))
_sample_order_mode = os.environ.get("PP_SAMPLE_ORDER", "auto")
_SORT_MIN_SAMPLES = 1 << 18


def set_sample_order(mode="auto"):
    """Processing order of the sampling points: "natural" (grid order),
    "sorted" (brick-major for 3-D grids, see pp_brick_order; source-sorted
    for 1-D / 2-D, see pp_sample_order) or "auto" (sorted for grids of at
    least 2^18 points).  Only the speed depends on it."""
    global _sample_order_mode
    if mode not in ("auto", "natural", "sorted"):
        raise ValueError(f"unknown sample order mode {mode}")
    _sample_order_mode = mode


class _OrderCache:
    """Sample orders of recently used grids.  An entry is valid while the
    grid tensor it was computed for is alive and unmodified (same storage
    pointer, version counter, sizes and strides) -- the forward and backward
    passes of a step then share one sort."""

    def __init__(self, size=4):
        self.size = size
        self.entries = []
        self.lock = threading.Lock()  # callers may run on several host threads

    @staticmethod
    def _key(grid, src):
        return (grid.data_ptr(), grid._version, tuple(grid.shape), tuple(grid.stride()),
                tuple(src), grid.device)

    def get(self, grid, src):
        key = self._key(grid, src)
        with self.lock:
            for i, (ref, k, perm) in enumerate(self.entries):
                if ref() is not None and k == key:
                    if i:
                        self.entries.insert(0, self.entries.pop(i))
                    return perm
        return None

    def put(self, grid, src, perm):
        with self.lock:
            self.entries = [e for e in self.entries if e[0]() is not None][: self.size - 1]
            self.entries.insert(0, (weakref.ref(grid), self._key(grid, src), perm))

    def clear(self):
        with self.lock:
            self.entries = []


_orders = _OrderCache()


def sample_order(grid, src_size):
    """Source-sorted processing order of `grid`'s sampling points (int32
    permutation) for a source of spatial size `src_size`."""
    L = _lib.load()
    src = (ctypes.c_int64 * len(src_size))(*[int(v) for v in src_size])
    d = _lib.desc(grid)
    nbytes = L.pp_sample_order_workspace_bytes(ctypes.byref(d), src)
    if nbytes == 0:
        raise RuntimeError(L.pp_last_error().decode(errors="replace"))
    nvox = grid.numel() // grid.shape[-1]
    perm = torch.empty(nvox, dtype=torch.int32, device=grid.device)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=grid.device)
    with _On(grid):
        _lib.check(L.pp_sample_order(ctypes.byref(d), src, ctypes.c_void_p(perm.data_ptr()),
                                     ctypes.c_void_p(ws.data_ptr()), nbytes, _lib.stream_of(grid)))
    return perm


def brick_order(grid, src_size):
    """Brick-major processing order of a 3-D grid's sampling points for a
    source of spatial size `src_size`: (perm, brick_start, records), int32
    device tensors and, for a float32 grid, the (samples, 4) float32 records
    of coordinates and indices in perm order (else None); see
    pp_brick_order."""
    L = _lib.load()
    src = (ctypes.c_int64 * 3)(*[int(v) for v in src_size])
    d = _lib.desc(grid)
    nbytes = L.pp_brick_order_workspace_bytes(ctypes.byref(d), src)
    nb = L.pp_brick_count(ctypes.byref(d), src)
    if nbytes == 0 or nb < 0:
        raise RuntimeError(L.pp_last_error().decode(errors="replace"))
    nvox = grid.numel() // grid.shape[-1]
    perm = torch.empty(nvox, dtype=torch.int32, device=grid.device)
    starts = torch.empty(nb + 1, dtype=torch.int32, device=grid.device)
    recs = torch.empty((nvox, 4), dtype=torch.float32, device=grid.device) if grid.dtype == torch.float32 else None
    ws = torch.empty(nbytes, dtype=torch.uint8, device=grid.device)
    with _On(grid):
        _lib.check(L.pp_brick_order(ctypes.byref(d), src, ctypes.c_void_p(perm.data_ptr()),
                                    ctypes.c_void_p(starts.data_ptr()),
                                    None if recs is None else ctypes.c_void_p(recs.data_ptr()),
                                    ctypes.c_void_p(ws.data_ptr()), nbytes, _lib.stream_of(grid)))
    return perm, starts, recs


def _brick_keys_fit(grid, src_size):
    """The brick sort keys (N * bricks * brick volume) fit in 32 bits."""
    nkeys = grid.shape[0] * _BRICK[0] * _BRICK[1] * _BRICK[2]
    for s, b in zip(src_size, _BRICK):
        nkeys *= -(-int(s) // b)
    return nkeys < (1 << 31)


_BRICK = (4, 4, 6)  # PP_BRICK_X, PP_BRICK_Y, PP_BRICK_Z


def _order_for(grid, src_size):
    """(perm, brick_start, records) for the call, or Nones for the natural
    order.  3-D grids get the brick-major order (it also drives the brick
    kernels); 1-D / 2-D grids the source-sorted one."""
    mode = _sample_order_mode
    if mode == "natural":
        return None, None, None
    nvox = grid.numel() // grid.shape[-1]
    if mode == "auto" and nvox < _SORT_MIN_SAMPLES:
        return None, None, None
    if nvox >= (1 << 31):
        return None, None, None
    bricks = grid.dim() == 5 and _brick_keys_fit(grid, src_size)
    entry = _orders.get(grid, src_size)
    if entry is None:
        entry = brick_order(grid, src_size) if bricks else (sample_order(grid, src_size), None, None)
        _orders.put(grid, src_size, entry)
    return entry


def set_deterministic(flag=True):
    """Make push / count (and the push halves of backward passes) bit-stable
    run to run: exact, order-independent accumulation."""
    global _deterministic
    _deterministic = bool(flag)


def get_deterministic():
    return _deterministic


# --------------------------------------------------------------------- #
# checks (pushpull.cpp:19-72)                                           #
# --------------------------------------------------------------------- #

def _fail(msg):
    raise RuntimeError("(): " + msg)


def _check_defined(t, name):
    if t is None:
        _fail(f"expected {name} not be undefined, but it is")
    if t.layout != torch.strided:
        _fail(f"expected {name}to have torch.strided layout, but it has {t.layout}")


def _check_123d(t, name):
    if t.dim() not in (3, 4, 5):
        _fail(f"expected 3D, 4D or 5D {name} but got input with sizes {list(t.shape)}")


def _check_not_empty(t, name):
    for i in range(2, t.dim()):
        if t.shape[i] <= 0:
            _fail(f"expected {name} to have non-empty spatial dimensions, but input has "
                  f"sizes {list(t.shape)} with dimension {i} being empty")


def _check_grid(grid):
    _check_defined(grid, "grid")
    _check_123d(grid, "grid")
    if grid.shape[-1] != grid.dim() - 2:
        _fail(f"expected grid to have size {grid.dim() - 2} in last dimension, but got grid "
              f"with sizes {list(grid.shape)}")
    _check_not_empty(grid, "grid")


def _check_pair(input, grid):
    _check_defined(input, "input")
    _check_defined(grid, "grid")
    if input.device != grid.device:
        _fail(f"expected input_opt and grid_opt to be on same device, but input_opt is on "
              f"{input.device} and grid_opt is on {grid.device}")
    ok = input.dtype == grid.dtype or (
        input.dtype in (torch.bfloat16, torch.float16) and grid.dtype == torch.float32)
    if not ok:
        _fail(f"expected input_opt and grid_opt to have the same dtype, but input_opt has "
              f"{input.dtype} and grid_opt has {grid.dtype}")
    _check_123d(input, "input")
    _check_grid(grid)
    _check_not_empty(input, "input")
    if input.dim() != grid.dim():
        _fail(f"expected input and grid to have the same number of dimensions, but got "
              f"{list(input.shape)} and {list(grid.shape)}")
    if input.dtype not in _FLOATS:
        _fail(f"expected a floating point input, got {input.dtype}")


def _check_opts(bound, interpolation):
    if not bound:
        _fail("expected non empty parameter bound_mode")
    if not interpolation:
        _fail("expected non empty parameter interpolation_mode")


def _require_cuda(t):
    if not t.is_cuda:
        raise RuntimeError("(): nitorch_b200 has no CPU backend: expected CUDA tensors, "
                           f"got a tensor on {t.device}")


def _grid32(grid):
    """Grids are float32 (float64 for float64 images)."""
    if grid.dtype in (torch.float16, torch.bfloat16):
        return grid.float()
    return grid


def _opts(bound, interpolation, extrapolate, grid=None, src_size=None):
    _check_opts(bound, interpolation)
    perm, starts, recs = (_order_for(grid, src_size) if grid is not None and grid.is_cuda
                          else (None, None, None))
    o = _lib.options([int(b) for b in bound], [int(i) for i in interpolation],
                     int(extrapolate), _lib.PP_DETERMINISTIC if _deterministic else 0,
                     None if perm is None else perm.data_ptr(),
                     None if starts is None else starts.data_ptr(),
                     None if recs is None else recs.data_ptr())
    o._keep = (perm, starts, recs)  # keep the order alive for the call
    return o


class _On:
    """Make `t`'s device current for the duration of a launch."""
    __slots__ = ("dev", "prev")

    def __init__(self, t):
        self.dev = t.device.index
        self.prev = None

    def __enter__(self):
        cur = torch.cuda.current_device()
        if self.dev is not None and cur != self.dev:
            self.prev = cur
            torch.cuda.set_device(self.dev)

    def __exit__(self, *exc):
        if self.prev is not None:
            torch.cuda.set_device(self.prev)


def _workspace(out):
    L = _lib.load()
    n = L.pp_push_workspace_bytes(ctypes.byref(_lib.desc(out)),
                                  _lib.PP_DETERMINISTIC if _deterministic else 0)
    if not n:
        return None, 0
    return torch.empty(n, dtype=torch.uint8, device=out.device), n


def _wsptr(ws):
    return None if ws is None else ctypes.c_void_p(ws.data_ptr())


# --------------------------------------------------------------------- #
# pull                                                                  #
# --------------------------------------------------------------------- #

def grid_pull(input, grid, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    out = torch.empty((grid.shape[0], input.shape[1], *grid.shape[1:-1]),
                      dtype=input.dtype, device=input.device)
    with _On(input):
        _lib.check(L.pp_grid_pull(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
                                  ctypes.byref(_lib.desc(out)), ctypes.byref(opt),
                                  _lib.stream_of(input)))
    return out


def grid_pull_backward(grad, input, grid, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    gi = torch.empty_like(input, memory_format=torch.contiguous_format) if input.requires_grad else None
    gg = torch.empty(g.shape, dtype=g.dtype, device=g.device) if grid.requires_grad else None
    ws, nws = _workspace(gi) if gi is not None else (None, 0)
    with _On(input):
        _lib.check(L.pp_grid_pull_backward(
            ctypes.byref(_lib.desc(grad)), ctypes.byref(_lib.desc(input)),
            ctypes.byref(_lib.desc(g)), _lib.ref(_lib.desc(gi)), _lib.ref(_lib.desc(gg)),
            ctypes.byref(opt), _lib.stream_of(input), _wsptr(ws), nws))
    out = []
    if gi is not None:
        out.append(gi)
    if gg is not None:
        out.append(gg.to(grid.dtype))
    return out


# --------------------------------------------------------------------- #
# push                                                                  #
# --------------------------------------------------------------------- #

def _push_shape(shape, ref_shape, dim):
    shape = list(shape) if shape is not None else []
    if not shape:
        return list(ref_shape)
    if len(shape) != dim:
        _fail(f"expected {dim + 2}source_size elements but got {len(shape)}")
    return [int(s) for s in shape]


def grid_push(input, grid, shape, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    dim = grid.dim() - 2
    if not (input.shape[0] == grid.shape[0] and list(input.shape[2:]) == list(grid.shape[1:-1])):
        _fail(f"expected input and grid to have same batch, width, height and (optionally) depth "
              f"sizes, but got input with sizes{list(input.shape)} and grid with sizes "
              f"{list(grid.shape)}")
    _check_opts(bound, interpolation)
    _require_cuda(input)
    shape = _push_shape(shape, input.shape[2:], dim)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, shape)
    out = torch.empty((grid.shape[0], input.shape[1], *shape), dtype=input.dtype, device=input.device)
    ws, nws = _workspace(out)
    with _On(input):
        _lib.check(L.pp_grid_push(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
                                  ctypes.byref(_lib.desc(out)), ctypes.byref(opt),
                                  _lib.stream_of(input), _wsptr(ws), nws))
    return out


def grid_push_backward(grad, input, grid, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, grad.shape[2:])
    gi = torch.empty_like(input, memory_format=torch.contiguous_format) if input.requires_grad else None
    gg = torch.empty(g.shape, dtype=g.dtype, device=g.device) if grid.requires_grad else None
    with _On(input):
        _lib.check(L.pp_grid_push_backward(
            ctypes.byref(_lib.desc(grad)), ctypes.byref(_lib.desc(input)),
            ctypes.byref(_lib.desc(g)), _lib.ref(_lib.desc(gi)), _lib.ref(_lib.desc(gg)),
            ctypes.byref(opt), _lib.stream_of(input)))
    out = []
    if gi is not None:
        out.append(gi)
    if gg is not None:
        out.append(gg.to(grid.dtype))
    return out


# --------------------------------------------------------------------- #
# count                                                                 #
# --------------------------------------------------------------------- #

def grid_count(grid, shape, bound, interpolation, extrapolate):
    _check_grid(grid)
    _check_opts(bound, interpolation)
    _require_cuda(grid)
    dim = grid.dim() - 2
    shape = _push_shape(shape, grid.shape[1:-1], dim)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, shape)
    out = torch.empty((grid.shape[0], 1, *shape), dtype=g.dtype, device=grid.device)
    ws, nws = _workspace(out)
    with _On(grid):
        _lib.check(L.pp_grid_count(ctypes.byref(_lib.desc(g)), ctypes.byref(_lib.desc(out)),
                                   ctypes.byref(opt), _lib.stream_of(grid), _wsptr(ws), nws))
    return out.to(grid.dtype)


def grid_count_backward(grad, grid, bound, interpolation, extrapolate):
    _check_grid(grid)
    _check_opts(bound, interpolation)
    _require_cuda(grid)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, grad.shape[2:])
    gg = torch.empty(g.shape, dtype=g.dtype, device=g.device)
    gr = grad.to(g.dtype)
    with _On(grid):
        _lib.check(L.pp_grid_count_backward(ctypes.byref(_lib.desc(gr)), ctypes.byref(_lib.desc(g)),
                                            ctypes.byref(_lib.desc(gg)), ctypes.byref(opt),
                                            _lib.stream_of(grid)))
    return gg.to(grid.dtype)


# --------------------------------------------------------------------- #
# spatial gradients                                                     #
# --------------------------------------------------------------------- #

def grid_grad(input, grid, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    dim = grid.dim() - 2
    out = torch.empty((grid.shape[0], input.shape[1], *grid.shape[1:-1], dim),
                      dtype=input.dtype, device=input.device)
    with _On(input):
        _lib.check(L.pp_grid_grad(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
                                  ctypes.byref(_lib.desc(out)), ctypes.byref(opt),
                                  _lib.stream_of(input)))
    return out


def grid_pull_grad(input, grid, bound, interpolation, extrapolate):
    """grid_pull and grid_grad of the same input and grid from one pass over
    the taps (pp_grid_pull_grad): [pulled (N, C, *grid), grad (N, C, *grid,
    D)]."""
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    dim = grid.dim() - 2
    out = torch.empty((grid.shape[0], input.shape[1], *grid.shape[1:-1]), dtype=input.dtype,
                      device=input.device)
    og = torch.empty((*out.shape, dim), dtype=input.dtype, device=input.device)
    with _On(input):
        _lib.check(L.pp_grid_pull_grad(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
                                       ctypes.byref(_lib.desc(out)), ctypes.byref(_lib.desc(og)),
                                       ctypes.byref(opt), _lib.stream_of(input)))
    return [out, og]


def grid_grad_backward(grad, input, grid, bound, interpolation, extrapolate):
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    gi = torch.empty_like(input, memory_format=torch.contiguous_format) if input.requires_grad else None
    gg = torch.empty(g.shape, dtype=g.dtype, device=g.device) if grid.requires_grad else None
    ws, nws = _workspace(gi) if gi is not None else (None, 0)
    with _On(input):
        _lib.check(L.pp_grid_grad_backward(
            ctypes.byref(_lib.desc(grad)), ctypes.byref(_lib.desc(input)),
            ctypes.byref(_lib.desc(g)), _lib.ref(_lib.desc(gi)), _lib.ref(_lib.desc(gg)),
            ctypes.byref(opt), _lib.stream_of(input), _wsptr(ws), nws))
    out = []
    if gi is not None:
        out.append(gi)
    if gg is not None:
        out.append(gg.to(grid.dtype))
    return out


# --------------------------------------------------------------------- #
# fused push(pull(.)) -- the normal operator P^T P                      #
# --------------------------------------------------------------------- #

def grid_pull_push(input, grid, bound, interpolation, extrapolate):
    """push(pull(input, grid), grid) onto the input's lattice in one pass:
    the result of grid_pull followed by grid_push with the input's spatial
    shape (up to summation order).  Not in the reference."""
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    out = torch.empty_like(input, memory_format=torch.contiguous_format)
    ws, nws = _workspace(out)
    with _On(input):
        _lib.check(L.pp_grid_pull_push(ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
                                       ctypes.byref(_lib.desc(out)), ctypes.byref(opt), _lib.stream_of(input),
                                       _wsptr(ws), nws))
    return out


def grid_pull_push_backward(grad, input, grid, bound, interpolation, extrapolate):
    """Gradients of grid_pull_push w.r.t. the input (P^T P grad: the operator
    is self-adjoint) and the grid, as requested by `requires_grad` (same
    conventions as grid_pull_backward)."""
    _check_pair(input, grid)
    _check_opts(bound, interpolation)
    _require_cuda(input)
    L = _lib.load()
    g = _grid32(grid)
    opt = _opts(bound, interpolation, extrapolate, g, input.shape[2:])
    if grad.stride() != input.stride():
        # the fused backward reads grad with the input's layout
        grad = torch.empty_strided(input.shape, input.stride(), dtype=grad.dtype,
                                   device=grad.device).copy_(grad)
    gi = torch.empty_like(input, memory_format=torch.contiguous_format) if input.requires_grad else None
    gg = torch.empty(g.shape, dtype=g.dtype, device=g.device) if grid.requires_grad else None
    ws, nws = _workspace(gi) if gi is not None else (None, 0)
    with _On(input):
        _lib.check(L.pp_grid_pull_push_backward(
            ctypes.byref(_lib.desc(grad)), ctypes.byref(_lib.desc(input)), ctypes.byref(_lib.desc(g)),
            _lib.ref(_lib.desc(gi)), _lib.ref(_lib.desc(gg)), ctypes.byref(opt), _lib.stream_of(input),
            _wsptr(ws), nws))
    out = []
    if gi is not None:
        out.append(gi)
    if gg is not None:
        out.append(gg.to(grid.dtype))
    return out


# The native multigrid resampling of the same compiled module, resolved on
# first use (nitorch_b200.multires imports this module's launch helpers).
from .enums import GridAlignType  # noqa: E402

_MULTIRES = ("fmg_prolongation", "fmg_restriction", "prolongation", "prolongation_backward", "resize",
             "resize_backward", "restriction", "restriction_backward")


def __getattr__(name):
    if name in _MULTIRES:
        from . import multires
        return getattr(multires, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
