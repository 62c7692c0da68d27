"""Batched simulations (xfd_batch_*): several independent scenes of uneven
sizes advanced together must give, per scene, the fields of the same scene run
alone through xfd_run -- bit for bit, in the persistent work-queue form (8-
and 16-row tiles) and the launch-per-phase form, since every node goes through
the same arithmetic in the same order -- and the alone run matches the oracle
(FP64 relative L2 <= 1e-12).  Random incidence angles
(theta, phi, psi) exercise the TFSF projection on every face."""
import numpy as np
import pytest

from oracle.reference_model import RefSimulation
from xfdtd_core_b200 import scene as S
from xfdtd_core_b200.engine import Batch, EngineError
from xfdtd_core_b200.host import SceneRun
from tests.scenes import dispersive_small, sphere_small

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _scenes(steps, sizes=(26, 33, 40, 47), seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        out.append(S.batched_sphere(n=n, radius_cells=float(rng.uniform(0.1, 0.3)) * n,
                                    eps_r=float(rng.uniform(2, 10)),
                                    theta=float(rng.uniform(0, np.pi)),
                                    phi=float(rng.uniform(0, 2 * np.pi)),
                                    psi=float(rng.uniform(0, 2 * np.pi)),
                                    pml=6, tfsf_start=9, steps=steps))
    return out


def _alone(scenes, precision, opts=None):
    got = []
    for sc in scenes:
        r = SceneRun(sc, precision=precision, options=opts)
        r.run()
        got.append(r.fields())
        r.close()
    return got


# (queue, tile rows): the persistent work-queue launch with 8- and 16-row
# tiles, and the launch per phase and form
FORMS = [(1, 8), (1, 16), (0, 8)]


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("depth", [4, 16])
@pytest.mark.parametrize("queue,rows", FORMS, ids=["queue8", "queue16", "launches"])
def test_batch_equals_alone_runs(precision, depth, queue, rows):
    steps = 70
    scenes = _scenes(steps)
    # the marching sweep alone (small lattices default to the split sweep)
    want = _alone(scenes, precision, {"march_ichunk": depth, "kernel": 4})
    runs = [SceneRun(sc, precision=precision) for sc in scenes]
    b = Batch([r.engine_handle() for r in runs],
              {"queue": queue, "tile_rows": rows, "march_ichunk": depth, "graph_chunk": 16})
    assert b.size() == len(scenes)
    b.run(33)  # two graph chunks and one single step
    b.run(steps - 33)
    b.sync()
    if queue:
        assert b.launches_per_step() == 1
    else:
        # per phase <= 6 tile lists (box forms, CPML tiles by slab axis) +
        # faces + 2 TFSF groups, and the step counters
        assert b.launches_per_step() <= 19
    for r, w in zip(runs, want):
        r.finish()
        for c, (g, ww) in enumerate(zip(r.fields(), w)):
            assert np.array_equal(g, ww), (r.n, c, float(np.max(np.abs(g - ww))))
    b.close()
    for r in runs:
        r.close()


def test_random_angle_scene_matches_oracle():
    sc = _scenes(90, sizes=(37,), seed=11)[0]
    orc = RefSimulation(sc)
    orc.run()
    r = SceneRun(sc)
    runs = [r, SceneRun(_scenes(90, sizes=(29,), seed=12)[0])]
    b = Batch([x.engine_handle() for x in runs])
    b.run(90)
    b.sync()
    r.finish()
    want = orc.e + orc.h
    ref = max(np.linalg.norm(w) for w in want)
    errs = [float(np.linalg.norm(g - w) / ref) for g, w in zip(r.fields(), want)]
    assert max(errs) <= TOL64, errs
    b.close()
    for x in runs:
        x.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_batch_autotune_keeps_results(precision):
    steps = 60
    scenes = _scenes(steps, sizes=(30, 45), seed=7)
    want = _alone(scenes, precision)
    runs = [SceneRun(sc, precision=precision) for sc in scenes]
    b = Batch([r.engine_handle() for r in runs], {"autotune": 3})
    b.run(steps)  # 12 x (1 + 3) tuning steps inside
    b.sync()
    tune = b.tuning_shapes()
    assert [t[:3] for t in tune] == ([(1, r, d) for r in (8, 16) for d in (8, 16, 32, 64)] +
                                     [(0, 8, d) for d in (8, 16, 32, 64)])
    assert all(t[3] > 0 for t in tune)
    best = min(tune, key=lambda t: t[3])
    assert (b.get_option("queue"), b.get_option("tile_rows"),
            b.get_option("march_ichunk")) == best[:3]
    assert [d for d, _ in b.tuning()] == [t[2] for t in tune]
    assert b.get_option("autotune") == 0
    tol = 1e-12 if precision == 0 else 1e-6
    for r, w in zip(runs, want):
        r.finish()
        got = r.fields()
        ref = max(np.linalg.norm(x) for x in w)
        err = max(float(np.linalg.norm(g - x) / ref) for g, x in zip(got, w))
        assert err <= tol, err
    b.close()
    for r in runs:
        r.close()


def test_batch_rejects_unbatched_features_and_mixed_precision():
    a = SceneRun(_scenes(10, sizes=(26,))[0], precision=0)
    c = SceneRun(_scenes(10, sizes=(26,))[0], precision=1)
    d = SceneRun(dispersive_small(steps=10), precision=0)  # ADE + NF2FF
    m = SceneRun(sphere_small(steps=10), precision=0)      # movie
    with pytest.raises(EngineError, match="INVALID_ARGUMENT"):
        Batch([a.engine_handle(), c.engine_handle()])
    with pytest.raises(EngineError, match="UNSUPPORTED"):
        Batch([a.engine_handle(), d.engine_handle()])
    with pytest.raises(EngineError, match="UNSUPPORTED"):
        Batch([m.engine_handle()])
    with pytest.raises(EngineError, match="twice"):
        Batch([a.engine_handle(), a.engine_handle()])
    b = Batch([a.engine_handle()])
    with pytest.raises(EngineError, match="n_steps"):
        b.run(11)
    with pytest.raises(EngineError, match="unknown option"):
        b.set_option("tile", 3)
    with pytest.raises(EngineError, match="tile_rows"):
        b.set_option("tile_rows", 12)
    b.set_option("queue", 0)
    with pytest.raises(EngineError, match="UNSUPPORTED"):
        b.set_option("tile_rows", 16)
    b.close()
    for x in (a, c, d, m):
        x.close()
