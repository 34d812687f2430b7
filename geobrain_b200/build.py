"""Build the in-tree CUDA library for sm_100a with nvcc.

    python -m geobrain_b200.build

produces ``geobrain_b200/_so/libgeobrain_b200.so`` (C ABI of
include/geobrain_b200.h, static CUDA runtime, no framework dependency).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# the translation units of the library (headers are included from them)
SRC = [os.path.join(HERE, "csrc", f) for f in ("gb_capi.cu", "gb_capi3d.cu")]
OUT = os.path.join(HERE, "_so", "libgeobrain_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    csrc = os.path.join(HERE, "csrc")
    return [os.path.join(csrc, f) for f in sorted(os.listdir(csrc))] + [
        os.path.join(ROOT, "include", "geobrain_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", OUT + ".tmp", *SRC]
    if verbose:
        cmd.append("-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
