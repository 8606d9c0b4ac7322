"""Build recipe for the reference's own C++ CPU backend (test infrastructure).

This compiles nitorch's ``_C`` extension from the reference sources, where
they lie, into ``oracle/_ref/`` (git-ignored; it travels with the tree).
Nothing is copied from the reference: the sources are compiled in place.

Sources: ``nitorch/_C/spatial.cpp`` (pybind module), ``nitorch/_C/src/*.cpp``
(native front-ends) and ``nitorch/_C/src/impl/*.cpp`` (kernels compiled for
the CPU namespace).  The flags follow the reference's own CPU build
(``setup_cext.py``): OpenMP parallel backend, ``NI_TORCH_VERSION`` for the
torch version guards.  Plain ``-fopenmp`` linking fails in this image
(no ``libgomp.spec``), so torch's bundled ``libgomp.so.1`` is linked.

Usage: ``python oracle/build_ref.py [REFERENCE_ROOT]``.  Only the oracle,
the tests and the CPU-baseline leg of ``bench.py`` load the result.
"""
import glob
import os
import sys


def build(reference_root=None, verbose=False):
    import torch
    from torch.utils import cpp_extension
    root = reference_root or os.environ.get("NITORCH_REFERENCE", "/root/reference")
    csrc = os.path.join(root, "nitorch", "_C")
    if not os.path.isdir(csrc):
        raise FileNotFoundError(f"reference sources not found under {csrc}")
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(here, "_ref")
    os.makedirs(out, exist_ok=True)
    sources = ([os.path.join(csrc, "spatial.cpp")]
               + sorted(glob.glob(os.path.join(csrc, "src", "*.cpp")))
               + sorted(glob.glob(os.path.join(csrc, "src", "impl", "*.cpp"))))
    tv = torch.__version__.split("+")[0].split(".")
    ni_version = int(tv[0]) * 10000 + int(tv[1]) * 100 + int(tv[2])
    torch_lib = os.path.join(os.path.dirname(torch.__file__), "lib")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    mod = cpp_extension.load(
        name="spatial",
        sources=sources,
        extra_cflags=["-O3", "-DAT_PARALLEL_OPENMP=1", "-fopenmp",
                      f"-DNI_TORCH_VERSION={ni_version}"],
        extra_ldflags=[f"-L{torch_lib}", "-l:libgomp.so.1",
                       f"-Wl,-rpath,{torch_lib}"],
        build_directory=out,
        with_cuda=False,
        verbose=verbose,
    )
    return mod


if __name__ == "__main__":
    m = build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
    print("built", m.__file__)
