"""Build libtfim.so (CUDA kernels + C ABI, sm_100a) and the `tfim` command-line engine.

Outputs go to tensorfim_b200/_lib/ inside the source tree, so they travel with the
repository to the machine that runs them.  Usage: ``python -m tensorfim_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
LIB = os.path.join(LIB_DIR, "libtfim.so")
CLI = os.path.join(LIB_DIR, "tfim")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-I" + INCLUDE, "-I" + CSRC, "-diag-suppress", "177"]

CU_SOURCES = ["common.cu", "parse.cu", "ingest.cu", "count_lop3.cu", "count_b1.cu", "count_pairs.cu", "count_proj.cu", "count_tc.cu", "count_fam.cu", "count_gram.cu", "allfi.cu", "shard.cu", "count_static.cu", "mlp.cu", "mine.cu", "resident.cu", "abi.cu"]
HEADERS = [os.path.join(CSRC, "tfim_internal.h"), os.path.join(INCLUDE, "tfim.h")]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s, *HEADERS]):
            jobs.append([NVCC, *NVFLAGS, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcuda"], verbose)
    cli_src = os.path.join(CSRC, "tfim_cli.cpp")
    if force or _newer(CLI, [cli_src, LIB, *HEADERS]):
        _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, cli_src, "-o", CLI, "-L" + LIB_DIR, "-ltfim",
              "-Wl,-rpath,$ORIGIN", "-pthread"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
