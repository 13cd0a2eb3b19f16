"""Build recipe of libt2b.so (sm_100a) in-tree: nvcc, no JIT cache.

Every CUDA source is compiled with -gencode arch=compute_100a,code=sm_100a
-lineinfo and linked into t2-relion_b200/libt2b.so next to this file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libt2b.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["api.cu", "project.cu", "estep.cu", "diff2_tc.cu", "proposal.cu", "imageprep.cu", "recon.cu", "noalloc.cu", "sampling.cpp", "io.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "t2b.h"))
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if _stale(obj, src, deps):
            cmd = [NVCC] + ARCH + FLAGS + list(extra_flags) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
