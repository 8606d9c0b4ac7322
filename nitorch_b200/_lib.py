"""ctypes binding of the C ABI in ``include/nitorch_b200.h``.

The shared library ``nitorch_b200/_C/libnitorch_b200.so`` is built in-tree
(``python -m nitorch_b200.build`` or ``make -C nitorch_b200/csrc``).  There
is no CPU fallback: if the library is missing or no CUDA device is
available, the first call raises.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_C", "libnitorch_b200.so")

PP_OK = 0
PP_ERR_ARG = -1
PP_ERR_DTYPE = -2
PP_ERR_CUDA = -3
PP_ERR_UNSUPPORTED = -4
PP_ERR_WORKSPACE = -5
PP_ERR_TIMEOUT = -6

PP_FLOAT32, PP_FLOAT64, PP_BFLOAT16, PP_FLOAT16 = 0, 1, 2, 3
PP_DETERMINISTIC = 1
PP_MAX_DIM = 8

_DTYPES = {
    torch.float32: PP_FLOAT32,
    torch.float64: PP_FLOAT64,
    torch.bfloat16: PP_BFLOAT16,
    torch.float16: PP_FLOAT16,
}


class PPTensor(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("sizes", ctypes.c_int64 * PP_MAX_DIM),
        ("strides", ctypes.c_int64 * PP_MAX_DIM),
    ]


class PPOptions(ctypes.Structure):
    _fields_ = [
        ("nbound", ctypes.c_int32),
        ("bound", ctypes.c_int32 * 3),
        ("norder", ctypes.c_int32),
        ("order", ctypes.c_int32 * 3),
        ("extrapolate", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("sample_order", ctypes.c_void_p),
        ("brick_start", ctypes.c_void_p),
        ("brick_records", ctypes.c_void_p),
    ]


class PPBatchEntry(ctypes.Structure):
    _fields_ = [
        ("src", PPTensor), ("trgt", PPTensor), ("grid", PPTensor), ("out", PPTensor), ("gg", PPTensor),
        ("opt", PPOptions),
    ]


EXPORTS = (
    "pp_abi_version", "pp_last_error", "pp_kernel_launches", "pp_last_kernel", "pp_push_workspace_bytes",
    "pp_grid_pull", "pp_grid_pull_backward", "pp_grid_push",
    "pp_grid_push_backward", "pp_grid_count", "pp_grid_count_backward",
    "pp_grid_grad", "pp_grid_grad_backward", "pp_grid_pull_grad", "pp_spline_coeff",
    "pp_spline_coeff_nd", "pp_sample_order_workspace_bytes", "pp_sample_order",
    "pp_sample_order_noalloc", "pp_brick_count", "pp_brick_order_workspace_bytes", "pp_brick_order",
    "pp_grid_pull_push", "pp_grid_pull_push_backward",
    "pp_batch_plan_bytes", "pp_batch_scratch_bytes", "pp_batch_plan", "pp_batch_run",
    "pp_svf_compose", "pp_svf_compose_backward", "pp_svf_workspace_bytes", "pp_affine_pull", "pp_affine_push",
    "pp_affine_grad_workspace_bytes", "pp_affine_grad_matrix", "pp_resize", "pp_resize_status",
    "pp_fmg_prolongation", "pp_fmg_restriction",
    "pp_grid_jacobian", "pp_grid_jacobian_backward", "pp_jacobian_det",
    "pp_regulariser", "pp_regulariser_grid",
)

PP_BATCH_PULL, PP_BATCH_PUSH, PP_BATCH_PUSH_BACKWARD = 0, 2, 4
PP_BATCH_PULL_BACKWARD, PP_BATCH_PULL_PUSH, PP_BATCH_PULL_PUSH_BACKWARD = 5, 7, 8

_lib = None


def _declare(L):
    T = ctypes.POINTER(PPTensor)
    O = ctypes.POINTER(PPOptions)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    L.pp_abi_version.restype = ctypes.c_int
    L.pp_last_error.restype = ctypes.c_char_p
    L.pp_last_kernel.restype = ctypes.c_char_p
    L.pp_kernel_launches.restype = ctypes.c_ulonglong
    L.pp_push_workspace_bytes.argtypes = [T, ctypes.c_int32]
    L.pp_push_workspace_bytes.restype = sz
    L.pp_grid_pull.argtypes = [T, T, T, O, vp]
    L.pp_grid_pull_backward.argtypes = [T, T, T, T, T, O, vp, vp, sz]
    L.pp_grid_push.argtypes = [T, T, T, O, vp, vp, sz]
    L.pp_grid_push_backward.argtypes = [T, T, T, T, T, O, vp]
    L.pp_grid_count.argtypes = [T, T, O, vp, vp, sz]
    L.pp_grid_count_backward.argtypes = [T, T, T, O, vp]
    L.pp_grid_grad.argtypes = [T, T, T, O, vp]
    L.pp_grid_pull_grad.argtypes = [T, T, T, T, O, vp]
    L.pp_grid_grad_backward.argtypes = [T, T, T, T, T, O, vp, vp, sz]
    L.pp_grid_pull_push.argtypes = [T, T, T, O, vp, vp, sz]
    L.pp_grid_pull_push_backward.argtypes = [T, T, T, T, T, O, vp, vp, sz]
    DP = ctypes.POINTER(ctypes.c_double)
    i32 = ctypes.c_int32
    L.pp_grid_jacobian.argtypes = [T, T, T, i32, DP, i32, i32, vp]
    L.pp_grid_jacobian_backward.argtypes = [T, T, T, T, i32, DP, i32, i32, vp]
    L.pp_jacobian_det.argtypes = [T, T, T, T, vp]
    IP = ctypes.POINTER(ctypes.c_int32)
    L.pp_regulariser.argtypes = [T, T, T, T, DP, DP, DP, DP, IP, vp]
    d = ctypes.c_double
    L.pp_regulariser_grid.argtypes = [T, T, T, T, d, d, d, d, d, DP, IP, vp]
    L.pp_svf_compose.argtypes = [T, T, O, vp]
    L.pp_svf_compose_backward.argtypes = [T, T, T, O, vp, vp, sz]
    L.pp_svf_workspace_bytes.argtypes = [T, ctypes.c_int32]
    L.pp_svf_workspace_bytes.restype = sz
    L.pp_affine_pull.argtypes = [T, T, T, O, vp]
    L.pp_affine_push.argtypes = [T, T, T, O, vp, vp, sz]
    L.pp_affine_grad_workspace_bytes.argtypes = [T]
    L.pp_affine_grad_workspace_bytes.restype = sz
    L.pp_affine_grad_matrix.argtypes = [T, T, T, T, O, vp, vp, sz]
    D3 = ctypes.c_double * 3
    L.pp_resize.argtypes = [T, T, D3, D3, O, vp]
    L.pp_resize_status.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
    L.pp_fmg_prolongation.argtypes = [T, T, O, vp]
    L.pp_fmg_restriction.argtypes = [T, T, O, vp]
    L.pp_batch_plan_bytes.argtypes = [ctypes.c_int32]
    L.pp_batch_plan_bytes.restype = sz
    L.pp_batch_scratch_bytes.argtypes = [ctypes.POINTER(PPBatchEntry), ctypes.c_int32, ctypes.c_int32]
    L.pp_batch_scratch_bytes.restype = sz
    L.pp_batch_plan.argtypes = [ctypes.POINTER(PPBatchEntry), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                vp, sz, vp, sz]
    L.pp_batch_run.argtypes = [vp, vp]
    L.pp_spline_coeff.argtypes = [T, T, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp]
    L.pp_spline_coeff_nd.argtypes = [T, T, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                     ctypes.c_int32, vp]
    I64P = ctypes.POINTER(ctypes.c_int64)
    L.pp_sample_order_workspace_bytes.argtypes = [T, I64P]
    L.pp_sample_order_workspace_bytes.restype = sz
    L.pp_sample_order.argtypes = [T, I64P, vp, vp, sz, vp]
    L.pp_sample_order_noalloc.argtypes = [T, I64P, vp, vp]
    L.pp_brick_count.argtypes = [T, I64P]
    L.pp_brick_count.restype = ctypes.c_int64
    L.pp_brick_order_workspace_bytes.argtypes = [T, I64P]
    L.pp_brick_order_workspace_bytes.restype = sz
    L.pp_brick_order.argtypes = [T, I64P, vp, vp, vp, vp, sz, vp]
    for name in EXPORTS:
        if name not in ("pp_last_error", "pp_last_kernel", "pp_push_workspace_bytes", "pp_kernel_launches",
                        "pp_sample_order_workspace_bytes", "pp_batch_plan_bytes", "pp_batch_scratch_bytes",
                        "pp_affine_grad_workspace_bytes", "pp_brick_count", "pp_brick_order_workspace_bytes"):
            getattr(L, name).restype = ctypes.c_int
    return L


def load():
    """Load (once) and return the C library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"nitorch_b200: CUDA library not built ({LIB_PATH} missing); "
                "run `python -m nitorch_b200.build`")
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def kernel_launches():
    """Kernels launched by the library so far (process-wide counter)."""
    return int(load().pp_kernel_launches())


def last_kernel():
    """Kernel family / mode / order / channel block of the last push/pull
    launch on this thread (see pp_last_kernel)."""
    return load().pp_last_kernel().decode()


def check(rc):
    if rc != PP_OK:
        msg = load().pp_last_error().decode(errors="replace")
        if rc == PP_ERR_UNSUPPORTED and "not implemented" in msg:
            raise NotImplementedError(msg)
        raise RuntimeError(msg)


def desc(t):
    """pp_tensor view of a torch tensor (borrowed: keep `t` alive)."""
    if t is None:
        return None
    d = PPTensor()
    d.data = t.data_ptr() if t.numel() else None
    try:
        d.dtype = _DTYPES[t.dtype]
    except KeyError:
        raise RuntimeError(f"(): unsupported dtype {t.dtype}") from None
    nd = t.dim()
    if nd > PP_MAX_DIM:
        raise RuntimeError(f"(): too many dimensions ({nd})")
    d.ndim = nd
    d.sizes[:nd] = t.shape
    d.strides[:nd] = t.stride()
    return d


def ref(d):
    return None if d is None else ctypes.byref(d)


def options(bound, order, extrapolate, flags=0, sample_order=None, brick_start=None, brick_records=None):
    o = PPOptions()
    o.sample_order = sample_order
    o.brick_start = brick_start
    o.brick_records = brick_records
    b = [int(x) for x in bound][:3]
    i = [int(x) for x in order][:3]
    o.nbound = len(b)
    o.bound[:len(b)] = b
    o.norder = len(i)
    o.order[:len(i)] = i
    o.extrapolate = int(extrapolate)
    o.flags = int(flags)
    return o


def stream_of(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)
