"""Kernel-level parity: each CUDA kernel of the engine, driven through the C
ABI, against the oracle's restatement of the reference loops on the same
seeded inputs (tests/cases.py).  FP64 tolerance: relative L2 <= 1e-12 per
field component (the reference's FP64 path; the two sides differ only in
rounding order and FMA contraction).  FP32 form: <= 1e-5 after a few steps."""
import numpy as np
import pytest

from tests.cases import KernelCase, rel_l2
from xfdtd_core_b200 import scene as S

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


KERNELS = [pytest.param((0, None), id="split"), pytest.param((1, None), id="fused"),
           pytest.param((1, 3), id="fused-ichunk3"), pytest.param((2, None), id="fused-tma"),
           pytest.param((2, 3), id="fused-tma-ichunk3"), pytest.param((3, None), id="march"),
           pytest.param((3, 3), id="march-ichunk3"), pytest.param((4, None), id="march-tma"),
           pytest.param((4, 3), id="march-tma-ichunk3"), pytest.param((4, 1), id="march-tma-ichunk1"),
           pytest.param((5, None), id="fmarch"), pytest.param((5, 3), id="fmarch-ichunk3"),
           pytest.param((5, 1), id="fmarch-ichunk1"), pytest.param((6, None), id="fvec"),
           pytest.param((6, 3), id="fvec-ichunk3"), pytest.param((7, None), id="hyb"),
           pytest.param((7, 3), id="hyb-ichunk3"), pytest.param((7, 1), id="hyb-ichunk1")]


def _compare(case, steps, precision=0, tol=FP64_TOL, graph=True, kernel=(1, None)):
    orc = case.oracle()
    orc.run(steps)
    eng = case.engine(precision=precision, n_steps=max(steps, 8), kernel=kernel[0],
                      ichunk=kernel[1])
    eng.set_option("graph", int(graph))
    eng.run(steps)
    eng.sync()
    got = eng.download_fields()
    want = orc.e + orc.h
    errs = [rel_l2(got[c], want[c]) for c in range(6)]
    assert max(errs) <= tol, errs
    return eng, orc


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("seed", [0, 1])
def test_yee_cpml_fp64(seed, kernel):
    _compare(KernelCase(n=(9, 10, 11), seed=seed), steps=4, kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_yee_no_cpml_fp64(kernel):
    _compare(KernelCase(n=(12, 7, 9), seed=3, slabs=()), steps=3, kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_yee_large_tile_crossing_fp32(kernel):
    """Several tiles along j and k in the FP32 form."""
    case = KernelCase(n=(21, 40, 70), seed=15)
    orc = case.oracle()
    orc.run(3)
    eng = case.engine(precision=1, n_steps=8, kernel=kernel[0], ichunk=kernel[1])
    eng.run(3)
    eng.sync()
    got = eng.download_fields()
    errs = [rel_l2(got[c], (orc.e + orc.h)[c]) for c in range(6)]
    assert max(errs) <= 1e-5, errs


@pytest.mark.parametrize("kernel", [4, 5, 6, 7])
@pytest.mark.parametrize("ichunk", [3, 4])
@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, 1e-5)], ids=["fp64", "fp32"])
def test_interior_forms(kernel, ichunk, precision, tol):
    """A grid long enough along z that the CPML-free interior holds whole
    tiles (pairs of tiles for kernel 6), so the CPML-free forms of the
    marching sweeps (the fused box kernel for kernel 7) run next to their
    CPML forms."""
    _compare(KernelCase(n=(24, 20, 140), seed=16), steps=3, precision=precision, tol=tol,
             kernel=(kernel, ichunk))


@pytest.mark.parametrize("kernel", KERNELS)
def test_yee_large_tile_crossing_fp64(kernel):
    # Several (j, k) tiles and i-chunks: 40 x 20 x 70 nodes.
    _compare(KernelCase(n=(39, 19, 69), seed=14), steps=3, kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_yee_cpml_fp32(kernel):
    _compare(KernelCase(n=(9, 10, 11), seed=4), steps=3, precision=1, tol=1e-5, kernel=kernel)


@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4, 5, 6, 7])
def test_graph_matches_eager(kernel):
    c = KernelCase(n=(10, 9, 8), seed=5)
    a = c.engine(n_steps=64, kernel=kernel)
    a.set_option("graph", 1)
    a.set_option("graph_chunk", 8)
    a.run(40)
    b = c.engine(n_steps=64, kernel=kernel)
    b.set_option("graph", 0)
    b.run(40)
    fa, fb = a.download_fields(), b.download_fields()
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("kernel", KERNELS)
def test_tfsf_faces_fp64(kernel):
    sc = S.dielectric_sphere(steps=24, dl=0.35 / 16, radius=0.06, pml=4, tfsf_start=6,
                             movie_interval=0)
    from oracle.reference_model import RefSimulation
    r = RefSimulation(sc)
    # Let the pulse reach the box: start from the incident grid of late steps.
    case = KernelCase(n=(r.nx, r.ny, r.nz), seed=6, field_scale=1e-3)
    t = dict(r.tfsf)
    t["e_inc"] = np.ascontiguousarray(np.roll(t["e_inc"], -12, axis=0))
    t["h_inc"] = np.ascontiguousarray(np.roll(t["h_inc"], -12, axis=0))
    case.tfsf = t
    orc = case.oracle()
    orc.run(6)
    eng = case.engine(n_steps=24, kernel=kernel[0], ichunk=kernel[1])
    eng.run(6)
    eng.sync()
    got = eng.download_fields()
    want = orc.e + orc.h
    errs = [rel_l2(got[c], want[c]) for c in range(6)]
    assert max(errs) <= FP64_TOL, errs


@pytest.mark.parametrize("kernel", KERNELS)
def test_lumped_current_source_fp64(kernel):
    case = KernelCase(n=(9, 10, 11), seed=7)
    case.add_lumped(comp=2, s=(3, 4, 4), e=(5, 6, 6), n_steps=8)
    case.add_lumped(comp=0, s=(2, 2, 2), e=(3, 4, 3), n_steps=8)
    _compare(case, steps=5, kernel=kernel)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_ade_fp64(kind, kernel):
    case = KernelCase(n=(9, 10, 11), seed=8 + kind, slabs=())
    case.add_ade(kind=kind, n_poles=2, n_mat=3)
    _compare(case, steps=5, kernel=kernel)


def test_ade_fp32():
    case = KernelCase(n=(9, 10, 11), seed=12, slabs=())
    case.add_ade(kind=0, n_poles=1, n_mat=2)
    _compare(case, steps=3, precision=1, tol=1e-5)


def test_nf2ff_fp64():
    case = KernelCase(n=(10, 11, 12), seed=13)
    case.add_nf2ff(nf=3, nt=8, dist=2, batch=3)
    eng, orc = _compare(case, steps=7)
    got = eng.nf2ff()
    acc = orc.nf2ff["acc"]
    want = acc[0::2] + 1j * acc[1::2]
    assert got.shape == want.shape
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= FP64_TOL


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_programmatic_dependent_launch_leaves_results_bit_equal(precision):
    """Sweep 0 with programmatic dependent launch (the default on small
    lattices: each kernel of the step may launch while the one before it
    finishes, and waits for it at entry) gives the fields, the movie frames
    and the field-time probe of the plain launches bit for bit."""
    from xfdtd_core_b200.host import SceneRun
    from tests.scenes import sphere_small
    got = []
    for pdl in (0, 1):
        r = SceneRun(sphere_small(steps=60), precision=precision, options={"kernel": 0, "pdl": pdl})
        assert r.get_engine_option("pdl") == pdl
        r.run(37)
        r.run(23)
        r.finish()
        got.append(r.fields() + [r.movie(0), r.field_time(0)])
        r.close()
    for a, b in zip(*got):
        assert np.array_equal(a, b)
