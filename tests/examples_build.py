"""Builds the reference's own example programs, unmodified, against this
library's C++ drop-in headers (include/xfdtd/... at the reference's include
paths, include/xtensor_subset for <xtensor/...>) and links them to
libxfdtd_host.so / libxfd_engine.so.

The example sources are read in place from the reference tree (test
infrastructure: only this recipe names that path); the binaries go to
tests/_examples/, which git ignores but which travels with the source tree,
so that the GPU tests can run them where the reference sources are absent.

    python tests/examples_build.py [--reference DIR] [--force]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_examples")
INCLUDE = os.path.join(ROOT, "include")
SHIM = os.path.join(INCLUDE, "xtensor_subset")
LIBDIR = os.path.join(ROOT, "xfdtd_core_b200", "lib")
DEFAULT_REFERENCE = "/root/reference"

# The reference's 3-D examples (test/src/examples), by path below it.  The
# 1-D and 2-D ones (slab_refection_transmission: TFSF1D; cylinder_scatter_2d:
# TFSF2D) are outside the 3-D hot path this library implements.
EXAMPLES = {
    "benchmark": "benchmark.cpp",
    "dielectric_cube_scatter": "dielectric_cube_scatter.cpp",
    "dielectric_resonator_antenna": "dielectric_resonator_antenna.cpp",
    "dielectric_sphere_scatter": "dielectric_sphere_scatter.cpp",
    "half_wave_dipole": "half_wave_dipole.cpp",
    "inverted_f_antenna": "inverted_f_antenna.cpp",
    "microstrip_branch_line_coupler": "microstrip_branch_line_coupler.cpp",
    "microstrip_line": "microstrip_line.cpp",
    "microstrip_low_pass": "microstrip_low_pass.cpp",
    "quarter_wave_transformer": "quarter_wave_transformer.cpp",
    "rlc_circuit": "rlc_circuit.cpp",
    "simple_capacitor": "simple_capacitor.cpp",
    "simple_circuit": "simple_circuit.cpp",
    "debye_sphere_scatter": "dispersive_sphere_scatter/debye_sphere_scatter.cpp",
    "drude_sphere_scatter": "dispersive_sphere_scatter/drude_sphere_scatter.cpp",
    "lorentz_sphere_scatter": "dispersive_sphere_scatter/lorentz_sphere_scatter.cpp",
}
# The ones the GPU tests run (linked executables); the rest are compiled only.
LINKED = ("dielectric_sphere_scatter", "half_wave_dipole", "dielectric_cube_scatter",
          "drude_sphere_scatter", "microstrip_line")


def example_dir(ref: str = DEFAULT_REFERENCE) -> str:
    return os.path.join(ref, "test", "src", "examples")


def available(ref: str = DEFAULT_REFERENCE) -> bool:
    return os.path.isdir(example_dir(ref))


def compile_cmd(src: str, out: str | None) -> list:
    cmd = ["g++", "-std=c++20", "-O2", "-I" + INCLUDE, "-I" + SHIM]
    if out is None:
        return cmd + ["-fsyntax-only", src]
    # the libraries found next to the tree the binary sits in, wherever it is copied
    rpath = "$ORIGIN/" + os.path.relpath(LIBDIR, OUT)
    return cmd + [src, "-o", out, "-L" + LIBDIR, "-lxfdtd_host", "-lxfd_engine",
                  "-Wl,-rpath," + rpath]


def build(ref: str = DEFAULT_REFERENCE, force: bool = False) -> list:
    os.makedirs(OUT, exist_ok=True)
    built = []
    for name in LINKED:
        src = os.path.join(example_dir(ref), EXAMPLES[name])
        out = os.path.join(OUT, name)
        libs = [os.path.join(LIBDIR, "libxfdtd_host.so"), os.path.join(LIBDIR, "libxfd_engine.so"),
                os.path.join(INCLUDE, "xfdtd", "xfdtd.h"),
                os.path.join(SHIM, "xtensor", "xt_core.hpp")]
        if not force and os.path.exists(out) and all(
                os.path.getmtime(out) >= os.path.getmtime(p) for p in [src] + libs):
            built.append(out)
            continue
        subprocess.check_call(compile_cmd(src, out + ".tmp"))
        os.replace(out + ".tmp", out)
        built.append(out)
    return built


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    for p in build(a.reference, a.force):
        print(p)


if __name__ == "__main__":
    sys.exit(main())
