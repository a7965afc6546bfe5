"""Build ``libfastkpc_b200.so`` in-tree with nvcc for sm_100a.

    python -m fastkpc_b200.build            # incremental
    python -m fastkpc_b200.build --force    # rebuild everything

Objects go to ``fastkpc_b200/_build/``; the shared library is written next to
this file so it travels with the source tree.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfastkpc_b200.so")
SOURCES = ["hostla.cpp", "design.cpp", "capi.cpp", "orient.cpp", "runtime.cu", "kernels_fit.cu", "kernels_stat.cu", "kernels_tprs.cu", "kernels_geom.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build fastkpc_b200")
    return cand


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "fastkpc_b200.h"))
    return hs


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in _headers())
    objs = []
    rebuilt = False
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            continue
        cmd = [nvcc(), *ARCH, *COMMON, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        rebuilt = True
    if force or rebuilt or not os.path.exists(LIB):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
