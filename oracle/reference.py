"""Loaders for the reference implementation itself -- TEST INFRASTRUCTURE.

* ``load_compiled()``: the reference's own C++ CPU backend, compiled from the
  reference sources by ``oracle/build_ref.py`` into ``oracle/_ref/``
  (the module ``nitorch._C.spatial``).  Returns None when not built.
* ``load_compiled_cuda()``: the same module built with the reference's CUDA
  backend for sm_100a by ``oracle/build_ref_cuda.py`` (``oracle/_ref/cuda/``),
  used to time the reference's own GPU kernels beside this library's.
* ``load_spatial()``: the reference's own ``nitorch.spatial`` package,
  imported from the reference tree with the compiled CPU backend as
  ``nitorch._C.spatial`` and the vendored TorchScript package as
  ``interpol`` (the import shim: only where the reference tree is present).
* ``load_ts_coeff()``: the reference's vendored prefilter
  ``nitorch/_C/_ts/coeff.py`` imported from the reference tree, when that
  tree is present (only in the development container, never on a GPU box).

Only the tests, the golden-fixture generator and the CPU-baseline leg of the
benchmark use these.
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "spatial.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "cuda", "spatial_cuda.so")
REFERENCE_ROOT = os.environ.get("NITORCH_REFERENCE", "/root/reference")

_compiled = None
_compiled_cuda = None
_ts = None


def load_compiled():
    """The compiled reference module (``nitorch._C.spatial``) or None.  When
    the CUDA build is already loaded, that module (which carries the CPU
    backend too) is returned: the two builds register the same pybind11
    types and cannot both be loaded in one process."""
    global _compiled
    if _compiled is None and _compiled_cuda is not None:
        return _compiled_cuda
    if _compiled is None and os.path.exists(REF_SO):
        import torch  # noqa: F401  (the extension links against libtorch)
        spec = importlib.util.spec_from_file_location("spatial", REF_SO)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _compiled = mod
    return _compiled


def load_compiled_cuda():
    """The reference module with its CUDA backend (sm_100a) or None (also
    None when the CPU-only build is already loaded in this process)."""
    global _compiled_cuda
    if _compiled_cuda is None and _compiled is None and os.path.exists(REF_CUDA_SO):
        import torch  # noqa: F401
        spec = importlib.util.spec_from_file_location("spatial_cuda", REF_CUDA_SO)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _compiled_cuda = mod
    return _compiled_cuda


def load_ts_coeff():
    """The reference's vendored prefilter module, or None if the reference
    tree is absent.  Its package uses relative imports, so it is loaded as a
    package named ``_ref_interpol`` rooted at ``nitorch/_C/_ts``."""
    global _ts
    if _ts is None:
        root = os.path.join(REFERENCE_ROOT, "nitorch", "_C", "_ts")
        if not os.path.isdir(root):
            return None
        spec = importlib.util.spec_from_file_location(
            "_ref_interpol", os.path.join(root, "__init__.py"),
            submodule_search_locations=[root])
        pkg = importlib.util.module_from_spec(spec)
        sys.modules["_ref_interpol"] = pkg
        spec.loader.exec_module(pkg)
        _ts = sys.modules["_ref_interpol.coeff"]
    return _ts


_spatial = None


def load_spatial():
    """The reference's nitorch.spatial (Python layer over its compiled CPU
    backend), or None if the reference tree or the compiled backend is
    absent."""
    global _spatial
    if _spatial is not None:
        return _spatial
    ref = load_compiled()
    root = os.path.join(REFERENCE_ROOT, "nitorch", "_C", "_ts")
    if ref is None or not os.path.isdir(root):
        return None
    os.environ.setdefault("NI_COMPILED_BACKEND", "C")
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if "interpol" not in sys.modules:
            spec = importlib.util.spec_from_file_location("interpol", os.path.join(root, "__init__.py"),
                                                          submodule_search_locations=[root])
            pkg = importlib.util.module_from_spec(spec)
            sys.modules["interpol"] = pkg
            spec.loader.exec_module(pkg)
        sys.modules.setdefault("nitorch._C.spatial", ref)
        if REFERENCE_ROOT not in sys.path:
            sys.path.append(REFERENCE_ROOT)
        import nitorch.spatial as S  # noqa: E402
    _spatial = S
    return S
