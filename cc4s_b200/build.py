"""Builds the CUDA library libcc4s_b200.so in-tree for sm_100a."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcc4s_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["gemm_f64.cu", "split_gemm.cu", "ops_cuda.cu", "schedule.cpp", "ccsd_real.cpp",
           "ccsd_complex.cpp", "drccd.cpp", "driver.cpp", "abi.cpp", "energy_noalloc.cu",
           "triples.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    newest_header = max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
                        if f.endswith((".h", ".cuh")))
    newest_header = max(newest_header, os.path.getmtime(os.path.join(HERE, "..", "include", "cc4s_cc.h")))
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(path)
                and os.path.getmtime(obj) > newest_header):
            continue
        lang = [] if src.endswith(".cu") else ["-x", "cu"]
        cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", path, "-o", obj]
        if src == "gemm_f64.cu":
            cmd += ["-Xptxas", "-v"] if verbose else []
        subprocess.run(cmd, check=True)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
