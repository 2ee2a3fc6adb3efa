"""Compile libpmilos_b200.so for sm_100a with nvcc (in-tree, next to this package).

Each source compiles to its own object in parallel (p-milos_b200/_build/), then
one nvcc call links the shared library."""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                  # p-milos_b200/
CSRC = os.path.join(ROOT, "csrc")
OBJ = os.path.join(ROOT, "_build")
OUT = os.path.join(ROOT, "libpmilos_b200.so")
SOURCES = ("pm_kernels.cu", "pm_wide.cu", "pm_wide_x32.cu", "pm_wide_x64.cu", "pm_stream.cu", "pm_stream_zm.cu",
           "pm_noalloc.cu", "pm_fits.cu", "pm_host.cpp", "pm_server.cpp")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"
FLAGS = ["-std=c++17", "-O3", ARCH, "-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(ROOT), "include", "pmilos.h"))
    deps.append(os.path.abspath(__file__))  # the source list and flags
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
        cmd = [cc] + FLAGS + (["-Xptxas=-v"] if verbose else []) + ["-c", os.path.join(CSRC, src), "-o", obj]
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    subprocess.run([cc, ARCH, "-shared", "-o", OUT + ".tmp"] + objs, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
