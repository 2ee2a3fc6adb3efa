"""Compile libpmilos_b200.so for sm_100a with nvcc (in-tree, next to this package)."""
from __future__ import annotations

import os
import shutil
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                  # p-milos_b200/
CSRC = os.path.join(ROOT, "csrc")
OUT = os.path.join(ROOT, "libpmilos_b200.so")
SOURCES = ("pm_kernels.cu", "pm_host.cpp", "pm_noalloc.cu")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


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
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), "-std=c++17", "-O3", ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
           "-o", OUT + ".tmp"] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
