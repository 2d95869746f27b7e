"""Build liblipika_cuda.so in-tree with nvcc for sm_100a.

The library is compiled from lipika_b200/csrc: CUDA translation units with
`-gencode arch=compute_100a,code=sm_100a`, host C++ with g++ and
-ffp-contract=off (table construction must not fuse multiply-adds), linked
against the static CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblipika_cuda.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU = ["lpk_abi.cu", "lpk_kernels.cu", "lpk_split.cu", "lpk_batch.cu", "lpk_mlp.cu", "lpk_noalloc.cu", "lpk_traj.cu"]
CPP = ["lpk_host.cpp"]


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "lipika_cuda.h"),
        os.path.join(HERE, "..", "include", "lipika_scene.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs, cmds = [], []
    inc = ["-I" + os.path.join(HERE, "..", "include")]
    for f in CU:
        o = os.path.join(BUILD, f + ".o")
        extra = os.environ.get("LPK_NVCC_FLAGS", "").split()  # e.g. tile-shape sweeps
        cmds.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-Xptxas", "-v" if verbose else "-O3", *extra, *inc, "-c", os.path.join(CSRC, f), "-o", o])
        objs.append(o)
    for f in CPP:
        o = os.path.join(BUILD, f + ".o")
        cmds.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                     "-I/usr/local/cuda/include", *inc, "-c", os.path.join(CSRC, f), "-o", o])
        objs.append(o)
    # translation units compile independently: one process each, in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = OUT + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
