"""Builds tempestrenderer_b200/libsvf.so in-tree for sm_100a.

    python -m tempestrenderer_b200.build [--force]

CUDA translation units are compiled by nvcc for sm_100a only; the host C++
units by g++.  svf_layout.cpp holds arithmetic that must agree with the
reference's x86-64 build bit for bit, so it is compiled without fused
multiply-adds (-ffp-contract=off).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "libsvf.so")
BUILD = os.path.join(REPO, "_build", "svf")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

CU_SOURCES = ["svf_kernels.cu", "svf_lm.cu", "svf_init.cu", "svf_ndf_tc.cu", "svf_mlp.cu", "svf_btf.cu",
              "svf_error.cu", "svf_ms.cu"]
# per-file nvcc flags: the pseudo-volume BRDF rounds every float operation on its
# own (no fused multiply-adds), as the reference's x86-64 build does
CU_FLAGS = {"svf_ms.cu": ["-fmad=false"]}
CXX_SOURCES = {"svf_host.cpp": ["-O2", "-ffp-contract=off"], "svf_host_init.cpp": ["-O2", "-ffp-contract=off"],
               "svf_host_lm.cpp": ["-O2", "-ffp-contract=off"], "svf_host_fit.cpp": ["-O2", "-ffp-contract=off"],
               "svf_host_mlp.cpp": ["-O2", "-ffp-contract=off"], "svf_host_btf.cpp": ["-O2", "-ffp-contract=off"],
               "svf_host_ms.cpp": ["-O2", "-ffp-contract=off"],
               "svf_layout.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math"],
               "svf_btf_file.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math"], "svf_exr.cpp": ["-O2"]}
HEADERS = ["svf_internal.h", "svf_host.h", "svf_model.cuh", "svf_layout.h", "svf_btf_file.h"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-ccbin", CXX]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "svf.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [NVCC, *NVCC_FLAGS, *CU_FLAGS.get(src, []), "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    for src, flags in CXX_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [CXX, "-std=c++17", "-fPIC", "-Wall", *flags, f"-I{CUDA_HOME}/include", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _newer(OUT, objs):
        tmp = OUT + ".tmp"
        cmd = [CXX, "-shared", "-o", tmp, *objs, f"-L{CUDA_HOME}/lib64", "-lcudart_static", "-lrt", "-ldl",
               "-lpthread", "-Wl,--no-undefined"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        shutil.move(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
