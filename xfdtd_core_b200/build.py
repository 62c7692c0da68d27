"""Build recipe for the native libraries, in-tree.

* ``lib/libxfd_engine.so``  -- the CUDA engine (csrc/engine), compiled for
  sm_100a only, behind the C ABI in include/xfd_engine.h.
* ``lib/libxfdtd_host.so``  -- the C++20 xfdtd::Simulation host library
  (csrc/host), which computes the FP64 set-up data and drives the engine.

nvcc cross-compiles sm_100a without a GPU, so both build on the CPU-only
machine; the built .so files travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "lib")
ENGINE_SRC = os.path.join(PKG, "csrc", "engine")
HOST_SRC = os.path.join(PKG, "csrc", "host")
ENGINE_LIB = os.path.join(LIBDIR, "libxfd_engine.so")
HOST_LIB = os.path.join(LIBDIR, "libxfdtd_host.so")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def _cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _files(d: str, exts) -> list:
    out = []
    for root, _, names in os.walk(d):
        for n in names:
            if n.endswith(exts):
                out.append(os.path.join(root, n))
    return sorted(out)


def build_engine(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _files(ENGINE_SRC, (".cu", ".cuh", ".h")) + [os.path.join(INCLUDE, "xfd_engine.h")]
    if not force and not _newer(ENGINE_LIB, srcs):
        return ENGINE_LIB
    nvcc = os.path.join(_cuda_home(), "bin", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-I" + INCLUDE, "-o", ENGINE_LIB + ".tmp",
           os.path.join(ENGINE_SRC, "engine.cu"), os.path.join(ENGINE_SRC, "nf2ff_static.cu"),
           "-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    os.replace(ENGINE_LIB + ".tmp", ENGINE_LIB)
    return ENGINE_LIB


def build_host(force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    cpp = _files(HOST_SRC, (".cpp",))
    srcs = cpp + _files(HOST_SRC, (".h", ".hpp")) + _files(INCLUDE, (".h", ".hpp"))
    if not cpp:
        return ""
    if not force and not _newer(HOST_LIB, srcs + [ENGINE_LIB]):
        return HOST_LIB
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-fopenmp", "-Wall", "-Wextra",
           "-ffp-contract=off", "-I" + INCLUDE, "-I" + HOST_SRC, "-o", HOST_LIB + ".tmp", *cpp,
           "-L" + LIBDIR, "-lxfd_engine", "-Wl,-rpath,$ORIGIN"]
    subprocess.check_call(cmd)
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    return HOST_LIB


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ENGINE_LIB)
    print(HOST_LIB)
