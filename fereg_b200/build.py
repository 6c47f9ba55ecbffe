"""Builds fereg_b200/libfereg_b200.so for sm_100a with nvcc (in-tree, no JIT cache).

    python -m fereg_b200.build [--force]
"""

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfereg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fopenmp", "--expt-relaxed-constexpr",
                  "-ccbin", "/usr/bin/g++"]
SOURCES = ["structure.cpp", "amg.cpp", "absorber.cu", "session.cu", "server.cu", "prep.cu", "dstruct.cu", "slopes.cu", "capi.cu"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "fereg_b200.h"))
    return hs


def _compile(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    srcp = os.path.join(CSRC, src)
    newest = max(os.path.getmtime(p) for p in [srcp] + _headers())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, False
    cmd = [NVCC] + CUFLAGS + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", srcp, "-o", obj]
    if not src.endswith(".cu"):
        cmd = ["/usr/bin/g++", "-O3", "-std=c++17", "-fPIC", "-march=x86-64-v3", "-fopenmp", "-Wall", "-Wextra",
               "-I/usr/local/cuda/include", "-c", srcp, "-o", obj]
    subprocess.run(cmd, check=True)
    return obj, True


def build(force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), SOURCES))
    objs = [o for o, _ in results]
    relink = force or not os.path.exists(LIB) or any(c for _, c in results) or any(
        os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)
    if relink:
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lgomp"], check=True)
    if verbose:
        print(f"built {LIB}" if relink else f"up to date: {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
