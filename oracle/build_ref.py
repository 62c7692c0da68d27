"""Build recipe for oracle/_ref: the reference's own library, unmodified.

Test infrastructure: compiles every ``src/**/*.cpp`` of the reference
(EMinsight/XFDTD_CORE) from where it lies, with its public and private
include trees, against the project's xtensor subset
(``include/xtensor_subset``, standing in for xtensor <= 0.25, which the
reference needs and which is not installed here), MPI and TBB off, Release
flags as the reference's CMakeLists.txt gives them (``-O3``, ISO C++20, no
fast-math), and links ``oracle/ref_driver.cpp`` against it into
``oracle/_ref/xfd_ref_driver``.  The reference's sources are read in place
and never copied; every output goes under ``oracle/_ref/`` (git-ignored).

    python -m oracle.build_ref [--reference DIR] [--jobs N] [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
DRIVER = os.path.join(OUT, "xfd_ref_driver")
SHIM = os.path.join(ROOT, "include", "xtensor_subset")
DEFAULT_REFERENCE = "/root/reference"
CXXFLAGS = ["-std=c++20", "-O3", "-DNDEBUG", "-pthread", "-ffp-contract=off", "-w"]


def reference_available(ref: str = DEFAULT_REFERENCE) -> bool:
    return os.path.isdir(os.path.join(ref, "src"))


def sources(ref: str):
    out = []
    for root, _, names in os.walk(os.path.join(ref, "src")):
        for n in names:
            if n.endswith(".cpp"):
                out.append(os.path.join(root, n))
    return sorted(out)


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(ref: str = DEFAULT_REFERENCE, jobs: int = 0, force: bool = False) -> str:
    if not os.path.isdir(os.path.join(ref, "src")):
        raise FileNotFoundError(f"reference sources not found under {ref}")
    os.makedirs(OBJ, exist_ok=True)
    inc = ["-I" + os.path.join(ref, "include"), "-I" + os.path.join(ref, "src", "include"),
           "-I" + SHIM]
    shim_hdrs = [os.path.join(SHIM, "xtensor", "xt_core.hpp")]
    objs, jobs_list = [], []
    for src in sources(ref):
        rel = os.path.relpath(src, os.path.join(ref, "src")).replace(os.sep, "__")
        obj = os.path.join(OBJ, rel[:-4] + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + shim_hdrs):
            jobs_list.append(["g++", *CXXFLAGS, *inc, "-c", src, "-o", obj])
    drv_obj = os.path.join(OBJ, "ref_driver.o")
    drv_src = os.path.join(HERE, "ref_driver.cpp")
    if force or _newer(drv_obj, [drv_src] + shim_hdrs):
        jobs_list.append(["g++", *CXXFLAGS, *inc, "-c", drv_src, "-o", drv_obj])
    n = jobs or os.cpu_count() or 4
    with cf.ThreadPoolExecutor(max_workers=n) as ex:
        for cmd, r in zip(jobs_list, ex.map(lambda c: subprocess.run(c, capture_output=True,
                                                                     text=True), jobs_list)):
            if r.returncode != 0:
                raise RuntimeError(f"{' '.join(cmd)}\n{r.stderr[-4000:]}")
    if force or _newer(DRIVER, objs + [drv_obj]):
        subprocess.check_call(["g++", "-pthread", "-o", DRIVER + ".tmp", drv_obj, *objs])
        os.replace(DRIVER + ".tmp", DRIVER)
    return DRIVER


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.reference, a.jobs, a.force))


if __name__ == "__main__":
    sys.exit(main())
