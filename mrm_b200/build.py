"""Builds mrm_b200/libmrm_gpu.so (sm_100a) in-tree with nvcc.

    python -m mrm_b200.build [--force] [-v]

Every translation unit compiles in its own nvcc process (in parallel), then
one nvcc call links the shared library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libmrm_gpu.so")
OBJ = os.path.join(HERE, "_build")
# longest compiles first (the pool takes them in this order)
SOURCES = ([f"csrc/k_row_f32_v{v}_g{g}.cu" for g in (2, 1, 0) for v in range(5)] +
           [f"csrc/k_creg_v{v}.cu" for v in range(3)] + [f"csrc/k_row_f64_v{v}.cu" for v in range(3)] +
           [f"csrc/k_col_f32_v{v}.cu" for v in range(3)] + [f"csrc/k_col_f64_v{v}.cu" for v in range(2)] +
           ["csrc/mrm_gpu.cu", "csrc/k_col.cu", "csrc/k_row_split.cu"])
HEADERS = ["csrc/common.cuh", "csrc/fft.cuh", "csrc/kernels.cuh", "csrc/philox.cuh", "csrc/tensor.cuh",
           "csrc/tma.cuh", "csrc/launch.h", "csrc/k_row.inc", "csrc/k_col.inc", "csrc/colreg.cuh", "csrc/regfft.cuh", "csrc/k_creg.inc", "../include/mrm_gpu.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(rel: str) -> float:
    return os.path.getmtime(os.path.join(HERE, rel))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(_mtime(s) <= t for s in SOURCES + HEADERS)


def _obj(src: str) -> str:
    return os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))


def _compile(src: str, verbose: bool) -> str:
    out = _obj(src)
    cmd = [nvcc(), *FLAGS, "-c", os.path.join(HERE, src), "-o", out + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    newest_header = max(_mtime(h) for h in HEADERS)
    todo = [s for s in SOURCES
            if force or not os.path.exists(_obj(s))
            or os.path.getmtime(_obj(s)) < max(_mtime(s), newest_header)]
    jobs = jobs or max(1, min(len(todo) or 1, os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(jobs) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *[_obj(s) for s in SOURCES]]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
