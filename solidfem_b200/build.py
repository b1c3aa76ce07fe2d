"""Builds libsolidfem_b200.so in-tree for sm_100a (B200).

The CUDA sources are compiled with nvcc for compute_100a/sm_100a; assembly.cu, setup_device.cu and
mesh_device.cu additionally with -fmad=false so the FP64 stiffness and multigrid hierarchy are bit-identical to the
reference's serial loops. The host
C++ is compiled without multiply-add contraction for the same reason (setup must reproduce the
reference's aggregates and coarse matrices to the bit). Objects go to solidfem_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsolidfem_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-ccbin", CXX, "-Xcompiler", "-fPIC,-ffp-contract=off",
               "--expt-relaxed-constexpr"] + ARCH
CU_SOURCES = {
    "solve.cu": [],
    "assembly.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "setup_device.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],
    "mesh_device.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true"],
}
CPP_SOURCES = ["mesh.cpp", "setup.cpp", "study.cpp", "server.cpp", "system.cpp"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-Wno-unused-function", "-Wno-unused-variable", "-I" + os.path.join(CUDA, "include")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source that changed and links the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".h")]
    headers.append(os.path.join(HERE, "..", "include", "solidfem_b200.h"))
    objects, jobs = [], []
    for src, extra in CU_SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers) or ptxas_info:
            cmd = [NVCC, "-c", path, "-o", obj] + NVCC_COMMON + extra
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
        objects.append(obj)
    for src in CPP_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers):
            jobs.append([CXX, "-c", path, "-o", obj] + CXX_FLAGS)
        objects.append(obj)
    # The translation units are independent: compile them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        for f in [pool.submit(_run, cmd) for cmd in jobs]:
            f.result()
    if _stale(LIB, objects):
        cmd = [NVCC, "-shared", "-o", LIB] + objects + ARCH + ["-ccbin", CXX, "-Xcompiler", "-fopenmp",
                                                              "-lgomp", "-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
