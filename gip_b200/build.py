"""Builds ``gip_b200/libgipb200.so`` from ``gip_b200/csrc/*.cu`` for sm_100a with nvcc.

The library is built in-tree so it travels with the repository; ``python -m
gip_b200.build`` rebuilds it when a source is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgipb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
         "--expt-relaxed-constexpr",
         "-I", INCLUDE, "-I", CSRC]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]


def _needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources() + _headers())


HOST_SRC = os.path.join(HERE, "cavity_gen.c")
HOST_LIB = os.path.join(HERE, "libgipcavity.so")


def build_host(force: bool = False) -> str:
    """The host-side cavity filler (plain C, OpenMP)."""
    if force or not os.path.exists(HOST_LIB) or \
            os.path.getmtime(HOST_SRC) > os.path.getmtime(HOST_LIB):
        cmd = ["/usr/bin/gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-Wall", "-o",
               HOST_LIB + ".tmp", HOST_SRC]
        subprocess.check_call(cmd)
        os.replace(HOST_LIB + ".tmp", HOST_LIB)
    return HOST_LIB


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    build_host(force)
    if not force and not _needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
