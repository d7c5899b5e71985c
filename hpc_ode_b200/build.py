"""Build the sm_100a CUDA library in-tree.

``python -m hpc_ode_b200.build`` compiles ``csrc/b200ode.cu`` (kernels + C ABI)
into ``hpc_ode_b200/libb200ode.so`` with nvcc for ``sm_100a`` only, and the
C++ host integrator (``csrc/host``) into ``hpc_ode_b200/libb200ode_host.so``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libb200ode.so")
HOST_LIB = os.path.join(PKG, "libb200ode_host.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# translation units of libb200ode.so: kernels + integrate ABI, request loop
CU_SOURCES = ["b200ode.cu", "serve.cu"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    out = []
    for d, _, fs in os.walk(CSRC):
        for f in fs:
            if f.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp")):
                out.append(os.path.join(d, f))
    inc = os.path.join(ROOT, "include")
    out.extend(os.path.join(inc, f) for f in os.listdir(inc))
    return out


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in _sources() if os.path.exists(s))


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale(LIB):
        cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"),
               "-o", LIB + ".tmp", *(os.path.join(CSRC, f) for f in CU_SOURCES)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    host_src = os.path.join(CSRC, "host")
    if os.path.isdir(host_src):
        cpps = sorted(os.path.join(host_src, f) for f in os.listdir(host_src) if f.endswith(".cpp"))
        if cpps and (force or _stale(HOST_LIB)):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"),
                   "-o", HOST_LIB + ".tmp", *cpps, "-L", PKG, "-lb200ode", "-Wl,-rpath,$ORIGIN"]
            subprocess.run(cmd, check=True)
            os.replace(HOST_LIB + ".tmp", HOST_LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
