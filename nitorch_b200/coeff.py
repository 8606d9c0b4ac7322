"""Interpolating B-spline prefilter with the ``interpol.coeff`` interface.

nitorch imports its prefilter from the third-party ``interpol`` package
(``nitorch/_C/grid.py:4``; PyPI ``torch-interpol``, unpinned in
``setup.cfg:110``).  Its arithmetic is vendored in the reference as
``nitorch/_C/_ts/coeff.py`` (Unser's recursive filtering; SPM / Thevenaz
initial conditions).  These two functions keep that interface -- integer
bound codes of ``_ts/bounds.py:7-14`` (0 zero, 1 replicate, 2 dct1, 3 dct2,
4 dst1, 5 dst2, 6 dft), integer orders -- and run the CUDA kernel of
``csrc/coeff.cu``.  Like the reference, only zero/dct1, replicate/dct2 and
dft are implemented; other bounds raise ``NotImplementedError``
(``coeff.py:233-251``) unless the order is 0 or 1 (identity).
"""
import ctypes
from typing import List, Optional

import torch

from . import _lib


def _pad(x, n):
    x = list(x) if isinstance(x, (list, tuple)) else [x]
    if len(x) < n:
        x = x + x[-1:] * (n - len(x))
    return [int(v) for v in x[:n]]


def _require_cuda(t):
    if not t.is_cuda:
        raise RuntimeError("spline_coeff: nitorch_b200 has no CPU backend: expected a CUDA "
                           f"tensor, got a tensor on {t.device}")


def spline_coeff(inp, bound: int, order: int, dim: int = -1, inplace: bool = False):
    """Spline coefficients along one dimension (``_ts/coeff.py:285-310``)."""
    _require_cuda(inp)
    out = inp if inplace else torch.empty_like(inp)
    if inp.numel() == 0:
        return out
    L = _lib.load()
    with torch.cuda.device(inp.device):
        _lib.check(L.pp_spline_coeff(ctypes.byref(_lib.desc(inp)), ctypes.byref(_lib.desc(out)),
                                     int(bound), int(order), int(dim), _lib.stream_of(inp)))
    return out


def spline_coeff_nd(inp, bound: List[int], order: List[int], dim: Optional[int] = None,
                    inplace: bool = False):
    """Spline coefficients along the last ``dim`` dimensions
    (``_ts/coeff.py:314-344``)."""
    _require_cuda(inp)
    if dim is None:
        dim = inp.dim()
    out = inp if inplace else torch.empty_like(inp)
    if inp.numel() == 0:
        return out
    b = _pad(bound, max(dim, 1))
    o = _pad(order, max(dim, 1))
    B = (ctypes.c_int32 * len(b))(*b)
    O = (ctypes.c_int32 * len(o))(*o)
    L = _lib.load()
    with torch.cuda.device(inp.device):
        _lib.check(L.pp_spline_coeff_nd(ctypes.byref(_lib.desc(inp)), ctypes.byref(_lib.desc(out)),
                                        len(b), B, len(o), O, int(dim), _lib.stream_of(inp)))
    return out
