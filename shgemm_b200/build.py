"""Builds libshgemm_b200.so (sm_100a) in-tree with nvcc.

    python -m shgemm_b200.build          # or: python shgemm_b200/build.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libshgemm_b200.so")
SOURCES = ["shgemm_lib.cu", "shgemm_api.cpp", "shgemm_server.cpp"]
HEADERS = ["ptx.cuh", "shgemm_kernel.cuh", "shgemm_kernel_tm.cuh", "shgemm_kernel_tm2.cuh", "server_host.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files += [os.path.join(ROOT, "include", "shgemm_b200.h"),
              os.path.join(ROOT, "include", "shgemm", "shgemm.hpp")]
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=default", "-Xcompiler", "-pthread", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES] + ["-o", LIB + ".tmp"]
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(cmd, check=True, env=env)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
