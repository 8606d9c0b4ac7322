"""Build recipe for the reference's own CUDA push/pull backend, compiled for
sm_100a -- TEST AND MEASUREMENT INFRASTRUCTURE, never the product.

nitorch compiles the same kernel sources twice, once for the CPU and once
with nvcc (``-x cu``) for CUDA (``setup_cext.py:25-37,349-356``), and
``nitorch/_C/src/pushpull.cpp:7-11`` dispatches CUDA tensors to
``cuda::pushpull`` when ``NI_WITH_CUDA`` is defined.  This recipe builds
that configuration with torch's cpp_extension into ``oracle/_ref/cuda/``
(git-ignored; the built module travels to GPU hosts with the tree):

* the pybind module ``nitorch/_C/spatial.cpp`` and the front-ends
  ``nitorch/_C/src/*.cpp`` (CPU-only, as in a CPU build) except
  ``pushpull.cpp``, which is compiled with ``NI_WITH_CUDA``;
* ``nitorch/_C/src/impl/*.cpp`` for the CPU namespace;
* ``nitorch/_C/src/impl/pushpull_common.cpp`` once more through nvcc for
  the ``cuda`` namespace, ``-gencode arch=compute_100a,code=sm_100a``, with
  the reference's nvcc flags.

cpp_extension picks the compiler by file extension, so two one-line stubs
are generated in the build folder; each only ``#include``s a reference
source file where it lies (nothing is copied).  Only the tests and the
side-by-side timing script ``tests/perf_reference_cuda.py`` load the result.

Usage: ``python oracle/build_ref_cuda.py [REFERENCE_ROOT]``.
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
    out = os.path.join(here, "_ref", "cuda")
    gen = os.path.join(out, "gen")
    os.makedirs(gen, exist_ok=True)

    def stub(name, text):
        path = os.path.join(gen, name)
        if not os.path.exists(path) or open(path).read() != text:
            with open(path, "w") as f:
                f.write(text)
        return path

    front = stub("pushpull_front_cuda.cpp",
                 "#define NI_WITH_CUDA 1\n"
                 f"#include \"{os.path.join(csrc, 'src', 'pushpull.cpp')}\"\n")
    kern = stub("pushpull_common_cuda.cu",
                f"#include \"{os.path.join(csrc, 'src', 'impl', 'pushpull_common.cpp')}\"\n")
    fronts = [p for p in sorted(glob.glob(os.path.join(csrc, "src", "*.cpp")))
              if os.path.basename(p) != "pushpull.cpp"]
    sources = ([os.path.join(csrc, "spatial.cpp")] + fronts + [front]
               + sorted(glob.glob(os.path.join(csrc, "src", "impl", "*.cpp"))) + [kern])
    tv = torch.__version__.split("+")[0].split(".")
    ni_version = int(tv[0]) * 10000 + int(tv[1]) * 100 + int(tv[2])
    torch_lib = os.path.join(os.path.dirname(torch.__file__), "lib")
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    mod = cpp_extension.load(
        name="spatial_cuda",
        sources=sources,
        extra_cflags=["-O3", "-DAT_PARALLEL_OPENMP=1", "-fopenmp", f"-DNI_TORCH_VERSION={ni_version}",
                      f"-I{os.path.join(csrc, 'src')}"],
        extra_cuda_cflags=["-O3", "-gencode=arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr",
                           "-std=c++17", f"-DNI_TORCH_VERSION={ni_version}", "-DAT_PARALLEL_OPENMP=1",
                           f"-I{os.path.join(csrc, 'src')}", f"-I{os.path.join(csrc, 'src', 'impl')}"],
        extra_ldflags=[f"-L{torch_lib}", "-l:libgomp.so.1", f"-Wl,-rpath,{torch_lib}"],
        build_directory=out,
        with_cuda=True,
        verbose=verbose,
    )
    return mod


if __name__ == "__main__":
    m = build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
    print("built", m.__file__)
