"""Build the sm_100a engine library in-tree (pgm_jax_b200/_build/libpgm_b200.so) with nvcc."""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libpgm_b200.so")
SOURCES = [os.path.join(HERE, "csrc", n)
           for n in ("pgm_api.cu", "pgm_md.cu", "pgm_static.cu", "pgm_nn.cu", "pgm_pimd.cu", "pgm_mpnn.cu")]
DEPS = SOURCES + [
    os.path.join(HERE, "csrc", "pgm_device.cuh"),
    os.path.join(HERE, "csrc", "pgm_kernels.cuh"),
    os.path.join(HERE, "csrc", "pgm_nn.cuh"),
    os.path.join(HERE, "csrc", "pgm_tc.cuh"),
    os.path.join(os.path.dirname(HERE), "include", "pgm_b200.h"),
]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if it is missing or older than its sources; return its path."""
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [NVCC, *FLAGS, "-o", LIB, *SOURCES, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
