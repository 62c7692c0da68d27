"""include/xfd_setup.h, the helpers a reference maintainer uses to hand a
Simulation's 18 update-coefficient arrays to the engine: buildClasses
factors them into the class table and per-node classes, and the arrays
rebuilt from (table, classes, curl factors) -- what the engine's sweeps
multiply out -- equal the input to the last bit or one rounding; a
coefficient whose curl terms are scaled unequally shows in the residual.
buildCurlFactors gives 1 / (size x kappa) per axis."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from tests.cases import KernelCase
from xfdtd_core_b200.engine import comp_shape

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("setup") / "probe.so")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I",
                           os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "setup_probe.cpp"), "-o", out])
    return ctypes.CDLL(out)


def _ptrs(arrs):
    keep = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
    return keep, (ctypes.c_void_p * len(keep))(*[a.ctypes.data for a in keep])


def _reference_arrays(case):
    ce, ceh_a, ceh_b, ch, che_a, che_b = case.oracle_coefficients()
    out = []
    for c in range(3):
        out += [ce[c], ceh_a[c], ceh_b[c]]
    for c in range(3):
        out += [ch[c], che_a[c], che_b[c]]
    return out


def _build(lib, n, coef, fe, fh):
    n_arr = (ctypes.c_int * 3)(*n)
    keep_c, pc = _ptrs(coef)
    keep_e, pe = _ptrs(fe)
    keep_h, ph = _ptrs(fh)
    cap = 12 * 65536
    table = np.zeros(cap)
    nodes = np.zeros((n[0] + 1) * (n[1] + 1) * (n[2] + 1), dtype=np.uint16)
    res = ctypes.c_double()
    k = lib.probe_build_classes(n_arr, pc, pe, ph, table.ctypes.data_as(ctypes.c_void_p),
                                ctypes.c_longlong(cap), nodes.ctypes.data_as(ctypes.c_void_p),
                                ctypes.byref(res))
    assert k > 0
    return table[:12 * k].reshape(k, 12), nodes.reshape(n[0] + 1, n[1] + 1, n[2] + 1), res.value


@pytest.mark.parametrize("seed", [0, 1])
def test_build_classes_rebuilds_the_18_arrays(lib, seed):
    case = KernelCase(n=(9, 10, 11), n_classes=7, seed=seed)
    coef = _reference_arrays(case)
    table, nodes, residual = _build(lib, case.n, coef, case.fe, case.fh)
    assert residual <= 4e-16
    rebuilt = KernelCase.from_setup(type("S", (), dict(
        n=case.n, table=table, lattice_class=nodes, fe=case.fe, fh=case.fh, slabs=[],
        lumped=[], fields=case.fields))())
    for q, (got, want) in enumerate(zip(_reference_arrays(rebuilt), coef)):
        assert got.shape == want.shape
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= 4e-16 * scale, q
    # one class per distinct node row: no more than the boundary patterns
    # times the original classes
    assert len(table) <= 64 * 7


def test_build_classes_reports_unequal_curl_terms(lib):
    case = KernelCase(n=(9, 10, 11), n_classes=4, seed=3)
    coef = _reference_arrays(case)
    coef[10] = coef[10].copy()
    coef[10][4, 5, 6] *= 1.7  # chxey scaled alone, as a ThinWire does
    _, _, residual = _build(lib, case.n, coef, case.fe, case.fh)
    assert residual > 0.1


def test_build_curl_factors(lib):
    rng = np.random.default_rng(5)
    n = (6, 7, 8)
    h_size = [rng.uniform(0.5, 2, n[a] + 1) for a in range(3)]
    e_size = [rng.uniform(0.5, 2, n[a]) for a in range(3)]
    ke = [rng.uniform(1, 5, n[a] + 1) for a in range(3)]
    kh = [rng.uniform(1, 5, n[a]) for a in range(3)]
    fe = [np.zeros(n[a] + 1) for a in range(3)]
    fh = [np.zeros(n[a]) for a in range(3)]
    args = [_ptrs(x) for x in (h_size, e_size, ke, kh, fe, fh)]
    lib.probe_curl_factors((ctypes.c_int * 3)(*n), *[p for _, p in args])
    for a in range(3):
        np.testing.assert_array_equal(fe[a], 1.0 / (h_size[a] * ke[a]))
        np.testing.assert_array_equal(fh[a], 1.0 / (e_size[a] * kh[a]))
