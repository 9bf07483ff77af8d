"""Builds the CUDA library in-tree: paraexastolog_b200/_lib/libesl_b200.so (sm_100a).

    python -m paraexastolog_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libesl_b200.so")
CLI = os.path.join(OUT_DIR, "esl_cli")
SOURCES = ["capi.cu", "table.cu", "table_static.cu", "graph.cu", "solve.cu", "sweep.cu", "mlp.cu", "multi.cu", "model.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    headers = [os.path.join(CSRC, "esl_internal.h"), os.path.join(REPO, "include", "esl_b200.h")]
    flags = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-extended-lambda",
                    "-I" + os.path.join(REPO, "include"), "-I" + CSRC]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT_DIR, src + ".o")
        objs.append(obj)
        if not force and _newer(obj, [path] + headers):
            continue
        cmd = [nvcc()] + flags + (["-x", "cu"] if src.endswith(".cpp") else []) + ["-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not _newer(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    # the reference's command line over the C ABI
    cli_src = os.path.join(CSRC, "cli.cpp")
    if force or not _newer(CLI, [cli_src, LIB] + headers):
        cmd = [nvcc()] + ARCH + ["-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"), cli_src, "-o", CLI,
               "-L" + OUT_DIR, "-lesl_b200", "-lcudart", "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
