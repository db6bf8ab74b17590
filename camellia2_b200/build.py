"""Build recipe of the CUDA library (in-tree, sm_100a only).

    python -m camellia2_b200.build      # -> camellia2_b200/libdpg_b200.so
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", f) for f in ("dpg_host.cu", "dpg_kernel.cu", "dpg_maps.cu")]
OUT = os.path.join(HERE, "libdpg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def build(verbose=False):
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + SRC + ["-o", OUT, "-lcudart"]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(OUT)
