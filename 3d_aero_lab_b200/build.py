"""Build recipe of libaero3d.so (sm_100a) - invoked by __graft_entry__.build() and the tests.

All CUDA/C++ sources in csrc/ are compiled by nvcc into one in-tree shared library with a
plain C ABI (include/aero3d.h).  FP32 division and square root use the hardware
approximations (-prec-div=false -prec-sqrt=false, flush-to-zero); FP64 code is unaffected.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libaero3d.so")
SOURCES = ["runtime.cu", "grid.cpp", "geom.cu", "solver.cu", "stage_tma.cu", "stage_pair.cu", "batch.cu", "server.cpp",
           "reduce.cu", "sample.cu", "static_forces.cu", "interp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "-ftz=true", "-prec-div=false", "-prec-sqrt=false", "-fmad=true", "--expt-relaxed-constexpr"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(HERE, "..", "include", "aero3d.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compile every source for sm_100a into 3d_aero_lab_b200/libaero3d.so."""
    if not force and not stale():
        return LIB
    cmd = [nvcc()] + ARCH + FLAGS + list(extra) + ["-shared", "-o", LIB + ".tmp"] + sources() + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
