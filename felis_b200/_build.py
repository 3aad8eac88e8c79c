"""Builds the FELIS B200 library in-tree (felis_b200/_lib/libfelis_b200.so).

Every CUDA translation unit is compiled for sm_100a only.  The FP64 plain
path is compiled with --fmad=false (and host code with -ffp-contract=off) so
that no multiply-add is contracted: the kernels then evaluate the same
IEEE operations, in the same order, as the CPU restatement of the reference.  The mixed-precision ensemble
(batch.cu, k_batch.cu) is not bound to the restatement bit for bit: its
kernels keep the compiler's multiply-add contraction and use the fast FP32
division, square root and sin/cos.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIBNAME = "libfelis_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include")]

# (source, extra flags)
UNITS = [
    ("lib/api.cu", ["--fmad=false"]),
    ("lib/k_particles.cu", ["--fmad=false"]),
    ("lib/k_field.cu", ["--fmad=false"]),
    ("lib/k_load.cu", ["--fmad=false"]),
    ("lib/k_1d.cu", ["--fmad=false"]),
    ("lib/k_wake.cu", ["--fmad=false"]),
    ("lib/k_sort.cu", []),
    ("lib/batch.cu", []),
    ("lib/k_batch.cu", ["--use_fast_math"]),
    ("lib/mlp.cu", []),
    ("lib/k_mlp.cu", []),
    ("lib/k_gemm.cu", []),
    ("lib/k_mlp_fused.cu", []),
    ("host/config.cpp", []),
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _deps(src: str) -> list[str]:
    d = os.path.dirname(src)
    out = [src]
    for root in (os.path.join(CSRC, "lib"), CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(root):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(root, f))
    return out


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    jobs = []
    objs = []
    for rel, extra in UNITS:
        src = os.path.join(CSRC, rel)
        obj = os.path.join(OBJDIR, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(obj, _deps(src)):
            lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
            cmd = [cc, *lang, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for msg in ex.map(run, jobs):
            if verbose and msg:
                print(msg)
    lib = os.path.join(LIBDIR, LIBNAME)
    if force or jobs or not os.path.exists(lib):
        cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    import sys

    print(build(verbose=True, force="--force" in sys.argv))
