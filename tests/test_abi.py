"""The engine library loads and exports every entry point include/xfd_engine.h
declares (no compute call: this runs without a GPU)."""
import ctypes
import os
import re

from xfdtd_core_b200 import build, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(xfd\w*)\s*\(", text)))


def test_engine_exports_header_symbols():
    path = build.build_engine()
    lib = ctypes.CDLL(path)
    names = _declared("xfd_engine.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(engine.exported_symbols()) == names


def test_engine_built_for_sm100a_only():
    assert "compute_100a" in " ".join(build.NVCC_FLAGS)


def test_host_exports_header_symbols():
    from xfdtd_core_b200 import host
    build.build_host()
    lib = ctypes.CDLL(build.HOST_LIB)
    names = [n for n in _declared("xfdtd_host.h")]
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(host.exported_symbols()) == names
