"""Builds libtamc_b200.so (sm_100a) and the tamc_b200 / tamc_b200_pt_opt CLIs in-tree.

Steps: generate the glibc-expf exception table (a host C program compared
against this machine's glibc), embed it with an assembler .incbin, compile the
C++ host sources with g++ and the CUDA sources with nvcc for sm_100a, link a
shared library with the static CUDA runtime, then link the CLI against it.
Outputs: tamc_b200/libtamc_b200.so, tamc_b200/bin/tamc_b200 and
tamc_b200/bin/tamc_b200_pt_opt (object files
under _build/ at the repository root).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SRC = os.path.join(PKG, "csrc")
OUT = os.path.join(ROOT, "_build", "tamc_b200")
LIB = os.path.join(PKG, "libtamc_b200.so")
CLI = os.path.join(PKG, "bin", "tamc_b200")
PT_OPT_CLI = os.path.join(PKG, "bin", "tamc_b200_pt_opt")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
GCC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["ctx.cu", "ref_kernels.cu", "fast_sa.cu", "sa_api.cu", "sa_noalloc.cu", "pt.cu", "fast_pt.cu",
              "fast_host.cu", "serve.cu", "gla.cu"]
CPP_SOURCES = ["host_instance.cpp", "method.cpp", "writers.cpp", "pt_opt.cpp"]
HEADERS = ["device.cuh", "expf_exact.h", "internal.h", "fast_common.cuh", "fast_sa.cuh", "fast_pt.cuh", "pt.cuh",
           "ref_kernels.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "tamc_gpu.h")]
    # 1. expf exception table
    gen = os.path.join(OUT, "gen_expf_table")
    table = os.path.join(OUT, "expf_table.bin")
    gsrc = os.path.join(SRC, "gen_expf_table.c")
    if _newer(gen, [gsrc, os.path.join(SRC, "expf_exact.h")]):
        _run([GCC, "-O2", "-ffp-contract=off", "-fopenmp", "-I", SRC, gsrc, "-o", gen, "-lm"])
    if _newer(table, [gen]):
        _run([gen, table])
    blob = os.path.join(OUT, "expf_blob.o")
    if _newer(blob, [table, os.path.join(SRC, "expf_blob.S")]):
        _run([GCC, "-c", f'-DEXPF_TABLE_BIN="{table}"', os.path.join(SRC, "expf_blob.S"), "-o", blob])
    # 2. objects
    steps = []
    objs = [blob]
    for s in CPP_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OUT, s + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdrs):
            steps.append([GXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                          "-I", SRC, "-c", src, "-o", obj])
    for s in CU_SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OUT, s + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdrs):
            steps.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                          "-Xcompiler", "-ffp-contract=off", "-I", SRC, "--expt-relaxed-constexpr",
                          "-Xptxas", "-warn-spills", "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(_run, steps))
    # 3. link
    if _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, "-lpthread", "-ldl", "-lrt"])
    for src_name, exe in (("cli.cpp", CLI), ("pt_opt_cli.cpp", PT_OPT_CLI)):
        obj = os.path.join(OUT, src_name + ".o")
        src = os.path.join(SRC, src_name)
        if _newer(obj, [src] + hdrs):
            _run([GXX, "-O2", "-std=c++17", "-ffp-contract=off", "-I", SRC, "-c", src, "-o", obj])
        if _newer(exe, [obj, LIB]):
            _run([GXX, "-o", exe, obj, LIB, "-Wl,-rpath,$ORIGIN/..", "-lpthread"])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
