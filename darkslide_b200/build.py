"""Build libdsgpu.so in-tree with nvcc for sm_100a.

Each translation unit gets its own flags: the demosaic, box-blur and scene
units are compiled with -fmad=false so that they round every product the way
the reference does; the NLM unit keeps FMA contraction.

    python -m darkslide_b200.build [--verbose]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdsgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "-I", INCLUDE, "-I", CSRC]

UNITS = [
    ("k_demosaic.cu", ["-fmad=false"]),
    ("k_box.cu", ["-fmad=false"]),
    ("k_scene.cu", ["-fmad=false", "-Xcompiler", "-ffp-contract=off"]),
    ("k_denoise.cu", ["-fmad=false"]),
    ("k_nlm.cu", []),
    ("k_peak.cu", []),
    ("k_cnn.cu", []),
    ("k_cnn_tc.cu", []),
    ("api.cu", []),
    ("batch.cu", []),
    ("noalloc.cu", []),
]


def _deps() -> list[str]:
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _deps() + [os.path.abspath(__file__)]
    objs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if ptxas_info or _stale(o, [s] + headers):
            cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, "-o", LIB, *objs, "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas-info" in sys.argv)
    print(LIB)
