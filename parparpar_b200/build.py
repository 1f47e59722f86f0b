"""Build the sm_100a shared library libparpar_b200.so in-tree with nvcc.

    python parparpar_b200/build.py   (not -m: importing the package loads the library)

Every CUDA translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo`` and linked into one
shared library next to this file, so the library travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libparpar_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")

SOURCES = [
    "gf16_kernels.cu",
    "gf16_tc.cu",
    "gf64_kernels.cu",
    "gf64_tc.cu",
    "gf64_fft.cu",
    "capi.cpp",
    "batch.cpp",
    "server.cpp",
    "noalloc.cu",
    "hash_kernels.cu",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "parpar_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _needs_build():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    cc = nvcc()
    objs = []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        cmd = [cc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
               "-I", os.path.join(HERE, "..", "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            cmd.append("-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([cc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
