"""Builds libjfem_gpu.so in-tree with nvcc for sm_100a (no JIT, no fallback).

Each translation unit is compiled to an object file under build/ (in
parallel), then the objects are linked into the shared library."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "libjfem_gpu.so")
SOURCES = ["jfg_matrix.cu", "jfg_mg.cu", "jfg_dense.cu", "jfg_krylov.cu", "jfg_api.cu", "jfg_noalloc.cu",
           "jfg_batch.cu", "jfg_cnn.cu", "jfg_cnn_tc.cu", "jfg_schwarz.cu", "jfg_block.cu",
           "jfg_spgemm.cu", "jfg_gs.cu", "jfg_assembly.cu",
           "jfg_cg_small.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [*ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "jfem_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in SOURCES]

    def compile_one(k):
        cmd = [NVCC, *FLAGS, "-c", "-o", objs[k], os.path.join(CSRC, SOURCES[k])]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd, cwd=CSRC)

    workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(workers) as ex:
        list(ex.map(compile_one, range(len(SOURCES))))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
