"""Build the engine's shared library in-tree with nvcc for sm_100a.

    python -m spectral_analyzer_b200.build

produces spectral_analyzer_b200/libacoustic_fdtd_b200.so from csrc/*.cu.
Host code is compiled without FMA contraction (-ffp-contract=off) so that the
create-time coefficient arithmetic rounds like the reference's.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_NAME = "libacoustic_fdtd_b200.so"
LIB_PATH = os.path.join(PKG, LIB_NAME)
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the engine")


def sources():
    return sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + glob.glob(os.path.join(PKG, "csrc", "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB_PATH
    cmd = [nvcc_path(), *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
           "-shared", "-I", os.path.join(ROOT, "include"),
           "-o", LIB_PATH + ".tmp", *sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
