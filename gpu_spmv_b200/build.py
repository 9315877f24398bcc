"""Build the engine library in-tree: ``python -m gpu_spmv_b200.build``.

Compiles every CUDA source for sm_100a (``-gencode arch=compute_100a,code=sm_100a``)
into ``gpu_spmv_b200/lib/libgpuspmv_b200.so``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int | None = None, quiet: bool = False) -> str:
    jobs = jobs or max(1, os.cpu_count() or 1)
    cmd = ["make", "-C", CSRC, f"-j{jobs}"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "lib", "libgpuspmv_b200.so")


if __name__ == "__main__":
    print(build(quiet="-q" in sys.argv))
