"""Build the CUDA library in-tree: ``python -m nitorch_b200.build``.

Compiles ``nitorch_b200/csrc/*.cu`` for sm_100a with nvcc (no GPU needed)
into ``nitorch_b200/_C/libnitorch_b200.so``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs=None, verbose=False):
    jobs = jobs or os.cpu_count() or 4
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    if not verbose:
        cmd.append("-s")
    subprocess.check_call(cmd)
    return os.path.join(HERE, "_C", "libnitorch_b200.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
