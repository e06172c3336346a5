"""Build the in-tree CUDA library ``libmicrocosmos_b200.so`` for sm_100a with nvcc.

    python -m microcosmos_b200.build

Compiles every ``csrc/*.cu`` into one shared library next to this file, with the
CUDA runtime linked statically (only the driver is needed at load time).  The
kernels are compiled with ``-fmad=false`` so that every product and sum is rounded
separately, as in the reference's float32 elementwise arithmetic.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmicrocosmos_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
         "-cudart", "static", "--expt-relaxed-constexpr"]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h"))
    return any(os.path.getmtime(f) > t for f in deps)


# Files that may be compiled with fused multiply-add contraction.  None: with contraction
# the dense pass drifts from the reference's separately rounded float32 ops by more than
# the 1e-5 rel-L2 bar after 100 steps of the 128x128 configuration (measured 1.1e-5).
FMA_FILES = ()


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in sources():
        flags = [f for f in FLAGS if f not in ("-shared",)]
        if os.path.basename(src) in FMA_FILES:
            flags = [f if f != "-fmad=false" else "-fmad=true" for f in flags]
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + ARCH + flags + list(extra) + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
        objs.append(obj)
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", LIB + ".tmp"] + objs
    if verbose:
        print(" ".join(cmd))
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
