"""Builds libps26119.so (the C-ABI engine library) in-tree: ps26119-solver_b200/lib/.

CUDA sources are compiled for sm_100a only, with -fmad=false (every a*b+c rounds twice, as
the reference's CPU build evaluates it); host C++ with -ffp-contract=off for the same reason.
Objects are rebuilt when a source or header is newer than the object.

    python ps26119-solver_b200/build.py [--force] [-j N]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libps26119.so")
CLI = os.path.join(LIB_DIR, "ps26119")  # the command-line tool
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

CU_SOURCES = ["engine.cu", "backend.cu", "batch.cu", "noalloc.cu"]
CPP_SOURCES = ["solver.cpp", "certify.cpp", "io.cpp", "serve.cpp", "c_api.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-Wall", "-Wextra",
             f"-I{CUDA}/include"]


def _headers():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    inc = os.path.join(ROOT, "include")
    out += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return out


def _stale(obj: str, src: str, headers: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def _compile(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(force: bool = False, jobs: int = 4, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    headers = _headers()
    cmds, objs = [], []
    for s in CU_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            cmds.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    for s in CPP_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            cmds.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        list(ex.map(_compile, cmds))
    if cmds or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _compile([NVCC, "-shared"] + ARCH + ["-o", LIB] + objs + ["-lpthread"])
    # the command-line tool, linked from the same objects
    cli_src, cli_obj = os.path.join(CSRC, "cli.cpp"), os.path.join(BUILD, "cli.cpp.o")
    if force or _stale(cli_obj, cli_src, headers):
        _compile(["g++"] + CXX_FLAGS + ["-c", cli_src, "-o", cli_obj])
    if not os.path.exists(CLI) or any(os.path.getmtime(o) > os.path.getmtime(CLI) for o in objs + [cli_obj]):
        _compile([NVCC] + ARCH + ["-o", CLI, cli_obj] + objs + ["-lpthread"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=4)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
