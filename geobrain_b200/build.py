"""Build the in-tree CUDA library for sm_100a with nvcc.

    python -m geobrain_b200.build [--force] [-v]

produces ``geobrain_b200/_so/libgeobrain_b200.so`` (C ABI of
include/geobrain_b200.h, static CUDA runtime, no framework dependency).
Every ``csrc/*.cu`` translation unit compiles to its own object, in
parallel; an object is rebuilt when its source or any header is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_so", "libgeobrain_b200.so")
OBJ = os.path.join(HERE, "_so", "obj")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def units():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))) + [
        os.path.join(ROOT, "include", "geobrain_b200.h")]


def sources():
    return units() + headers()


def _obj(cu: str) -> str:
    return os.path.join(OBJ, os.path.basename(cu)[:-3] + ".o")


def _stale(cu: str, t_headers: float) -> bool:
    o = _obj(cu)
    return not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(cu), t_headers)


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    t_h = max(os.path.getmtime(h) for h in headers())
    todo = [cu for cu in units() if force or _stale(cu, t_h)]

    def compile_one(cu: str):
        cmd = [nvcc(), *ARCH, *FLAGS, "-c", "-o", _obj(cu) + ".tmp", cu]
        if verbose:
            cmd.append("-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(_obj(cu) + ".tmp", _obj(cu))
        return cu, r

    failed = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for cu, r in ex.map(compile_one, todo):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                failed.append(os.path.basename(cu))
    if failed:
        raise RuntimeError(f"nvcc failed on {', '.join(failed)}")
    objs = [_obj(cu) for cu in units()]
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs], check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
