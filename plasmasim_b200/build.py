"""Builds the in-tree CUDA library plasmasim_b200/libplasmab200.so for sm_100a."""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libplasmab200.so")
SOURCES = [os.path.join(HERE, "csrc", "api.cu"), os.path.join(HERE, "csrc", "noalloc.cu"),
           os.path.join(HERE, "csrc", "pic2d.cu"), os.path.join(HERE, "csrc", "transport.cu")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.isfile(cand) else "nvcc"


def _newest_input() -> float:
    files = glob.glob(os.path.join(HERE, "csrc", "*")) + [os.path.join(ROOT, "include", "plasma_b200.h")]
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False, out: str = LIB, defines=()) -> str:
    """nvcc of the library sources for sm_100a into `out` (the in-tree
    library by default); `defines` are extra -D flags of a variant build."""
    if not force and os.path.isfile(out) and os.path.getmtime(out) >= _newest_input():
        return out
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(ROOT, "include"), *(f"-D{d}" for d in defines),
           "-o", out, *SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    if out == LIB:
        build_driver()
    return out


DRIVER = os.path.join(HERE, "pic3d_main")


def build_driver() -> str:
    """The C host driver (plasmasim_b200/driver/pic3d_main.c) linked to the library."""
    cmd = ["gcc", "-std=gnu11", "-O2", os.path.join(HERE, "driver", "pic3d_main.c"),
           "-I", os.path.join(ROOT, "include"), "-L", HERE, "-lplasmab200",
           f"-Wl,-rpath,{HERE}", "-Wl,-rpath,$ORIGIN", "-lm", "-o", DRIVER]
    subprocess.run(cmd, check=True)
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
