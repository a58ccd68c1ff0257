"""Build libopem_b200.so in-tree with nvcc for sm_100a.

Usage: python -m openparem_b200.build   (or build() from __graft_entry__)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libopem_b200.so")
SOURCES = ["basis.cpp", "topology.cpp", "dense.cpp", "assemble.cu", "krylov.cu", "lsq.cu", "mixed.cu", "patch_tc.cu", "engine.cu",
           "server.cu", "post.cpp", "project.cu", "port2d.cpp", "portfem.cpp", "estimate.cu", "refine.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-fopenmp,-O3", "--expt-relaxed-constexpr"]


def build(verbose=False, extra=()):
    objs = []
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(HERE, "_build", s + ".o")
        deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".h")]
        deps.append(os.path.join(HERE, "..", "include", "opem_b200.h"))
        if not os.path.exists(obj) or any(os.path.getmtime(d) > os.path.getmtime(obj) for d in deps):
            fl = list(FLAGS)
            if s in ("dense.cpp", "port2d.cpp"):
                # small dense complex LA: plain complex arithmetic, no C99 inf/NaN recovery
                fl[fl.index("-fPIC,-fopenmp,-O3")] = "-fPIC,-fopenmp,-O3,-fcx-limited-range"
            cmd = [NVCC] + fl + list(extra) + ["-x", "cu" if s.endswith(".cu") else "c++", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC] + FLAGS + ["-shared", "-o", LIB] + objs + ["-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
