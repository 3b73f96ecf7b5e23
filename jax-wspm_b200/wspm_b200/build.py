"""Build libwspm.so (hand-written sm_100a CUDA) in-tree with nvcc.

The library is compiled for ``sm_100a`` only (``-gencode
arch=compute_100a,code=sm_100a``) and written next to this file, so it
travels with the source tree.  cudart is linked statically.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG_ROOT), "include")
LIB = os.path.join(HERE, "libwspm.so")
SOURCES = ["assembly.cu", "krylov.cu", "picard.cu", "capi.cu", "transport.cu", "noalloc.cu", "ensemble.cu", "adjoint.cu", "precond.cu", "balance.cu", "pattern.cu", "measure.cu", "pattern_dev.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _inputs():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh"))]
    files.append(os.path.join(INCLUDE, "wspm.h"))
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build_library(force=False, verbose=False, extra_flags=()):
    """Compile every .cu in csrc/ into libwspm.so; returns the library path."""
    if not force and up_to_date():
        return LIB
    build_dir = os.path.join(PKG_ROOT, "_build")
    os.makedirs(build_dir, exist_ok=True)
    objs = [os.path.join(build_dir, src.replace(".cu", ".o")) for src in SOURCES]
    cmds = [[NVCC, *FLAGS, *extra_flags, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
            for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), file=sys.stderr)
    # translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static", *objs, "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
