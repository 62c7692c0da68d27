"""Failure detection on the GPU without a GPU fault.

* Bounded stage waits: with the "stage_wait_cycles" option at 1 cycle every
  TMA-staged sweep CTA gives up at its first wait for a staged plane (the
  bulk copy cannot land within a cycle), sets the error word, waits for its
  loads in flight with the default budget and returns -- no trap, no hang.
  xfd_sync (and xfd_batch_sync for batched engines) then reports
  XFD_ERR_TIMEOUT, and a new engine on the same CUDA context runs clean and
  matches the oracle.
* Bounded queue waits of the persistent batched kernel: with the test hook
  "queue_stall_test" one work item waits for a count that nothing reaches; after
  "queue_wait_cycles" it gives up, xfd_batch_sync reports XFD_ERR_TIMEOUT, and
  a new batch on the same context is bit-equal to the scenes run alone.
* The NaN / Inf watchdog ("watchdog_interval"): a field value set to NaN is
  reported by the next sync as XFD_ERR_NUMERIC; on clean fields the watchdog
  changes nothing (bit-equal fields) and the sync succeeds.
"""
import numpy as np
import pytest

from tests.cases import KernelCase, rel_l2
from tests.scenes import sphere_small
from xfdtd_core_b200.engine import Batch, EngineError
from xfdtd_core_b200.host import SceneRun

pytestmark = pytest.mark.gpu


def _box_case():
    # long along z so that sweep 7's fused interior box runs beside its CPML tiles
    return KernelCase(n=(24, 20, 140), seed=16)


@pytest.mark.parametrize("kernel", [4, 7])
def test_stage_wait_budget_reports_timeout_then_clean_engine_runs(kernel):
    case = _box_case()
    eng = case.engine(kernel=kernel, n_steps=16)
    assert eng.get_option("stage_wait_cycles") == 0
    eng.set_option("stage_wait_cycles", 1)
    eng.run(4)
    with pytest.raises(EngineError, match="TIMEOUT"):
        eng.sync()
    eng.close()
    # the context is intact: a fresh engine with the default budget is exact
    orc = case.oracle()
    orc.run(4)
    eng = case.engine(kernel=kernel, n_steps=16)
    eng.run(4)
    eng.sync()
    got = eng.download_fields()
    errs = [rel_l2(g, w) for g, w in zip(got, orc.e + orc.h)]
    assert max(errs) <= 1e-12, errs
    eng.close()


def test_batch_sync_reports_stage_timeout():
    from xfdtd_core_b200 import scene as S
    scenes = [S.batched_sphere(n=n, radius_cells=0.2 * n, eps_r=4.0, theta=0.3, phi=0.5,
                               psi=0.1, pml=6, tfsf_start=9, steps=20) for n in (40, 47)]
    runs = [SceneRun(sc, options={"stage_wait_cycles": 1}) for sc in scenes]
    b = Batch([r.engine_handle() for r in runs], {"graph_chunk": 4})
    b.run(4)
    with pytest.raises(EngineError, match="TIMEOUT"):
        b.sync()
    b.close()
    for r in runs:
        r.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_batch_queue_wait_reports_timeout_then_clean_batch_runs(precision):
    from xfdtd_core_b200 import scene as S
    scenes = [S.batched_sphere(n=n, radius_cells=0.2 * n, eps_r=4.0, theta=0.3, phi=0.5,
                               psi=0.1, pml=6, tfsf_start=9, steps=20) for n in (40, 33)]
    runs = [SceneRun(sc, precision=precision) for sc in scenes]
    b = Batch([r.engine_handle() for r in runs],
              {"queue": 1, "queue_stall_test": 1, "queue_wait_cycles": 2_000_000,
               "graph": 0})
    assert b.get_option("queue_wait_cycles") == 2_000_000
    b.run(2)
    with pytest.raises(EngineError, match="TIMEOUT"):
        b.sync()
    b.close()
    for r in runs:
        r.close()
    # the context is intact: a clean batch equals the scenes run alone
    want = []
    for sc in scenes:
        r = SceneRun(sc, precision=precision, options={"kernel": 4})
        r.run()
        want.append(r.fields())
        r.close()
    runs = [SceneRun(sc, precision=precision) for sc in scenes]
    b = Batch([r.engine_handle() for r in runs], {"queue": 1, "graph_chunk": 8})
    b.run(20)
    b.sync()
    for r, w in zip(runs, want):
        r.finish()
        for g, x in zip(r.fields(), w):
            assert np.array_equal(g, x)
    b.close()
    for r in runs:
        r.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_watchdog_reports_non_finite_field(precision):
    case = _box_case()
    eng = case.engine(precision=precision, kernel=None, n_steps=16)
    eng.set_option("watchdog_interval", 4)
    fields = [f.astype(eng.dtype) for f in case.fields]
    fields[4][12, 10, 70] = np.nan  # one interior Hy value
    eng.upload_fields(fields)
    eng.run(8)
    with pytest.raises(EngineError, match="NUMERIC"):
        eng.sync()
    eng.close()


def test_watchdog_on_clean_fields_changes_nothing():
    sc = sphere_small(steps=60)
    a = SceneRun(sc, options={"watchdog_interval": 5})
    a.run()
    b = SceneRun(sc)
    b.run()
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
    a.close()
    b.close()
