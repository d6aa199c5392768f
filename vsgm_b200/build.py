"""Build the native library in-tree: vsgm_b200/libvsgm_b200.so (+ the pm_pipeline driver
and the view_tools driver).

    python -m vsgm_b200.build [--force]

Host C++ is compiled with g++ (C++17, OpenMP), the engine with nvcc for sm_100a
only.  Objects go to vsgm_b200/_build/; a target is rebuilt when any source or
header is newer than it.
"""
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libvsgm_b200.so")
DRIVER = os.path.join(PKG, "pm_pipeline")
VIEW_TOOLS = os.path.join(PKG, "view_tools")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SRCS = ["planner.cpp", "graph.cpp", "capi_host.cpp"]
CUDA_SRCS = ["engine.cu", "mlp.cu", "partition.cu"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INC, "*.h"))


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps, force):
    return force or not os.path.exists(target) or os.path.getmtime(target) < _newest(deps)


def build(force=False, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in HOST_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + hdrs, force):
            _run(["g++", "-std=c++17", "-O3", "-fopenmp", "-fPIC", "-Wall", "-Wno-unused-function", f"-I{INC}", "-c", s, "-o", o])
        objs.append(o)
    for src in CUDA_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + hdrs, force):
            cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", f"-I{INC}", "-c", s, "-o", o]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(o)
    if _stale(LIB, objs, force):
        _run([NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-lgomp", "-Xlinker", "-rpath,$ORIGIN"])
    drv = os.path.join(CSRC, "pm_pipeline.cpp")
    if os.path.exists(drv) and _stale(DRIVER, [drv, LIB] + hdrs, force):
        _run(["g++", "-std=c++17", "-O3", "-fopenmp", f"-I{INC}", drv, "-o", DRIVER, f"-L{PKG}", "-lvsgm_b200",
              "-Wl,-rpath,$ORIGIN"])
    tools = os.path.join(CSRC, "view_tools.cpp")
    if os.path.exists(tools) and _stale(VIEW_TOOLS, [tools, LIB] + hdrs, force):
        _run(["g++", "-std=c++17", "-O3", f"-I{INC}", tools, "-o", VIEW_TOOLS, f"-L{PKG}", "-lvsgm_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
