"""Build libparw2v.so (CUDA, sm_100a) and the ``parw2v`` command-line tool, in-tree.

    python -m par_word2vec_b200.build [--force] [-v]

Outputs ``par_word2vec_b200/libparw2v.so`` and ``par_word2vec_b200/bin/parw2v``; objects go
to ``_build/`` at the repository root.  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libparw2v.so")
CLI = os.path.join(HERE, "bin", "parw2v")

CU_SOURCES = ["api.cu", "k_setup.cu", "k_det.cu", "k_pack.cu", "k_plain.cu", "k_batched.cu", "k_loss.cu", "k_walks.cu"]
CXX_SOURCES = ["frontend.cpp"]
HEADERS = ["common.cuh", "internal.h", "mma.cuh", "sentence.cuh", "bulk.cuh", "repel.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libparw2v")


def _cxx() -> str:
    # the image exports CXX as a wrapper GCC; the system g++ is the one nvcc also uses
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "parw2v.h")]
    jobs, objs = [], []
    for src in CU_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs + [__file__]):
            flags = list(NVCC_FLAGS)
            if ptxas_info and src.endswith(".cu"):
                flags += ["-Xptxas", "-v"]
            jobs.append([nvcc] + flags + ["-c", path, "-o", obj])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"], verbose)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB] + hdrs)):
        _run([_cxx(), "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), cli_src, "-o", CLI,
              "-L" + HERE, "-lparw2v", "-Wl,-rpath,$ORIGIN/..", "-lm"], verbose)
    return "\n".join(logs)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args(argv)
    out = build(a.force, a.verbose, a.ptxas_info)
    if a.ptxas_info:
        print(out)
    print(LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())
