"""The allocation-free NF2FF step, xfd_nf2ff_step_static, against the engine's
own NF2FF accumulation on the same seeded case.

The entry point exists for callers that cannot allocate device memory: an
FDTD loop inside a larger GPU application that owns all device memory
through its own pool or a fixed arena, where a cudaMalloc would fail or
would stall the device mid-loop.  It takes the caller's field arrays,
phasors and accumulator and keeps its per-step samples in a fixed scratch
array compiled into the library.  The test itself holds its buffers in
torch tensors (the test may allocate; the entry point does not) and calls
the entry point through the C ABI.

This file is named to be collected last, so that a run which stops at its
first failure has already run every other test."""
import numpy as np
import pytest

from tests.cases import KernelCase
from xfdtd_core_b200 import engine as E

TOL = 1e-12      # relative L2, the FP64 tolerance of the other parity tests
FP32_TOL = 1e-5  # relative L2, the FP32 kernel-case budget of the other parity tests
STEPS = 7
N_STEPS = 8


def _case():
    case = KernelCase(n=(10, 11, 12), seed=13)
    case.add_nf2ff(nf=3, nt=N_STEPS, dist=2, batch=3)
    return case


def _face_points(tasks):
    return [(e[0] - s[0]) * (e[1] - s[1]) * (e[2] - s[2]) for s, e in tasks]


def _face_order(acc, nf, tasks):
    """The entry point's (frequency, current q, point) layout reordered to
    the engine's xfd_get_nf2ff order (frequency, face, q, point of face)."""
    counts = _face_points(tasks)
    begin = np.concatenate([[0], np.cumsum(counts)])
    a = acc.reshape(nf, 4, int(begin[-1]))
    return np.concatenate([a[f, q, begin[d]:begin[d + 1]]
                           for f in range(nf) for d in range(6) for q in range(4)])


def _static_pass(torch, case, dev, precision=0, compensated=False):
    """Runs the case's fields step by step (FP64 or FP32 engine) and folds
    each step with the allocation-free entry point into a fresh zeroed
    accumulator (with a compensation array when `compensated`)."""
    nf = case.nf2ff
    eng = case.engine(precision=precision, n_steps=N_STEPS)
    te = torch.from_numpy(np.ascontiguousarray(nf["te"], dtype=np.float64)).to(dev)
    th = torch.from_numpy(np.ascontiguousarray(nf["th"], dtype=np.float64)).to(dev)
    P = sum(_face_points(nf["tasks"]))
    acc = torch.zeros(nf["nf"] * 4 * P * 2, dtype=torch.float64, device=dev)
    comp = torch.zeros_like(acc) if compensated else None
    stream = torch.cuda.current_stream(dev).cuda_stream
    for t in range(STEPS):
        eng.run(1)
        eng.sync()
        fields = [torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in eng.download_fields()]
        E.nf2ff_step_static(case.n, precision, [f.data_ptr() for f in fields], nf["tasks"],
                            te.data_ptr(), th.data_ptr(), nf["nf"], N_STEPS, t, nf["nf"],
                            acc.data_ptr(), stream=stream,
                            acc_comp_dev=comp.data_ptr() if compensated else 0)
        torch.cuda.synchronize(dev)
    a = acc.cpu().numpy()
    if compensated:
        a = a + comp.cpu().numpy()
    return _face_order(a[0::2] + 1j * a[1::2], nf["nf"], nf["tasks"])


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
def test_static_step_matches_engine_nf2ff_twice():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    case = _case()
    ref_eng = case.engine(n_steps=N_STEPS)
    ref_eng.run(STEPS)
    ref_eng.sync()
    want = ref_eng.nf2ff()
    first = _static_pass(torch, case, dev)
    second = _static_pass(torch, case, dev)  # the scratch holds the first pass's last step
    for got in (first, second):
        assert got.shape == want.shape
        assert _rel(got, want) <= TOL
    assert np.array_equal(first, second)


@pytest.mark.gpu
def test_static_step_matches_oracle_fp64_compensated():
    """The compensated form (acc + acc_comp) against the oracle's own NF2FF
    sums (the CPU restatement of calculateJ / calculateM), FP64."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    case = _case()
    orc = case.oracle()
    orc.run(STEPS)
    acc = orc.nf2ff["acc"]
    want = acc[0::2] + 1j * acc[1::2]
    got = _static_pass(torch, case, dev, compensated=True)
    assert got.shape == want.shape
    assert _rel(got, want) <= TOL


@pytest.mark.gpu
def test_static_step_fp32_fields_match_engine_fp32_twice():
    """FP32 fields (precision 1) into the FP64 sums, against the FP32
    engine's own NF2FF on the same case, on two passes in a row."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    case = _case()
    ref_eng = case.engine(precision=1, n_steps=N_STEPS)
    ref_eng.run(STEPS)
    ref_eng.sync()
    want = ref_eng.nf2ff()
    orc = case.oracle()
    orc.run(STEPS)
    acc = orc.nf2ff["acc"]
    want64 = acc[0::2] + 1j * acc[1::2]
    first = _static_pass(torch, case, dev, precision=1)
    second = _static_pass(torch, case, dev, precision=1)
    for got in (first, second):
        assert got.shape == want.shape
        assert _rel(got, want) <= TOL  # same FP32 fields, same FP64 sums
        assert _rel(got, want64) <= FP32_TOL
    assert np.array_equal(first, second)


def test_static_step_rejects_oversized_surface():
    """A surface above the scratch capacity is refused before anything is
    launched (no GPU needed)."""
    n = (600, 600, 600)
    tasks = [((1, 1, 1), (600, 600, 600))] + [None] * 5
    with pytest.raises(E.EngineError, match="exceeds the static scratch"):
        E.nf2ff_step_static(n, 0, [8] * 6, tasks, 8, 8, 1, 10, 0, 1.0, 8)
