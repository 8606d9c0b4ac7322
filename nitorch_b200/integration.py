"""Route an installed nitorch through this backend.

nitorch selects its compiled backend in ``nitorch/_C/grid.py:9-79`` by
importing ``grid_pull ... BoundType`` from the module ``nitorch._C.spatial``
(``NI_COMPILED_BACKEND=C``), and imports its prefilter from ``interpol``
(``grid.py:4-7``).  ``install()`` registers this package's modules under
those names *before* nitorch is imported, so ``nitorch.spatial.grid_*`` run
on the B200 kernels unmodified.
"""
import os
import sys
import types


def install(set_env=True):
    """Register ``nitorch._C.spatial`` (and ``interpol.coeff``) aliases.

    Must run before ``import nitorch``.  Returns the spatial module.
    """
    from . import coeff, spatial
    if set_env:
        os.environ["NI_COMPILED_BACKEND"] = "C"
    sys.modules["nitorch._C.spatial"] = spatial
    if "interpol" not in sys.modules:
        # Minimal interpol stand-in: the prefilter plus the names grid.py
        # imports from it (grid.py:4-7).
        from .enums import BoundType
        pkg = types.ModuleType("interpol")
        pkg.__path__ = []
        mcoeff = types.ModuleType("interpol.coeff")
        mcoeff.spline_coeff = coeff.spline_coeff
        mcoeff.spline_coeff_nd = coeff.spline_coeff_nd
        mpush = types.ModuleType("interpol.pushpull")
        mpush.grid_push = spatial.grid_push
        mbounds = types.ModuleType("interpol.bounds")
        import enum

        class _TSBoundType(enum.Enum):
            zero = zeros = 0
            replicate = nearest = 1
            dct1 = mirror = 2
            dct2 = reflect = 3
            dst1 = antimirror = 4
            dst2 = antireflect = 5
            dft = wrap = 6
        mbounds.BoundType = _TSBoundType
        msplines = types.ModuleType("interpol.splines")
        from .enums import InterpolationType
        msplines.InterpolationType = InterpolationType
        for name, m in (("coeff", mcoeff), ("pushpull", mpush), ("bounds", mbounds),
                        ("splines", msplines)):
            setattr(pkg, name, m)
            sys.modules[f"interpol.{name}"] = m
        sys.modules["interpol"] = pkg
        del BoundType
    return spatial


# nitorch.spatial callers of the push/pull path that this package also
# provides as fused CUDA implementations: name -> "module:function"
_CALLERS = {
    "exp": "svf:exp",
    "resize": "api:resize",
    "reslice": "api:reslice",
    "grid_jacobian": "jacobian:grid_jacobian",
    "grid_jacdet": "jacobian:grid_jacdet",
}


def patch_callers(spatial_module):
    """After ``install()`` and ``import nitorch.spatial as S``, route
    ``S.exp``, ``S.resize``, ``S.reslice``, ``S.grid_jacobian`` and
    ``S.grid_jacdet`` to this package's fused versions for CUDA tensors
    (velocity exponentiation with one kernel per squaring, affine sampling
    without a materialised grid, Jacobians in one pass).  Tensors on other
    devices keep nitorch's own functions (which, after ``install()``, still
    call this backend for their CUDA pulls).  Returns the patched names."""
    import importlib

    import torch

    patched = []
    for name, target in _CALLERS.items():
        original = getattr(spatial_module, name, None)
        if original is None or getattr(original, "_nitorch_b200", False):
            continue
        mod, fn = target.split(":")
        fast = getattr(importlib.import_module(f"{__package__}.{mod}"), fn)

        def dispatch(x, *args, _fast=fast, _orig=original, **kwargs):
            if isinstance(x, torch.Tensor) and x.is_cuda:
                return _fast(x, *args, **kwargs)
            return _orig(x, *args, **kwargs)
        dispatch.__name__ = name
        dispatch.__doc__ = (original.__doc__ or "") + f"\n(CUDA tensors: nitorch_b200.{mod}.{fn})"
        dispatch._nitorch_b200 = True
        setattr(spatial_module, name, dispatch)
        patched.append(name)
    return patched
