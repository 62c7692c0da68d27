"""The x-slab decomposition on the GPU: the slabs of a seeded lattice run as
separate engines (here all on one device; the same calls drive one engine
per GPU) that exchange their ghost planes' E_y, E_z through xfd_halo_copy
after every step.  The gathered owned values match the one-domain oracle
within 1e-12 (FP64) on every sweep, the fused box sweep 7 included (its
box lies inside each slab's local lattice) -- also with an oblique TFSF
plane wave (xfd_set_tfsf_slab: each engine cuts the global source to its
nodes) and ADE media cut by slab."""
import numpy as np
import pytest

from tests.cases import KernelCase, rel_l2, tfsf_source
from xfdtd_core_b200 import slab

pytestmark = pytest.mark.gpu
SLABS = ((0, True, 4), (0, False, 3), (1, True, 3), (1, False, 3), (2, True, 3), (2, False, 4))


def _case(n, steps):
    c = KernelCase(n=n, seed=33, slabs=SLABS)
    c.add_lumped(comp=2, s=(n[0] // 2 - 1, 4, 4), e=(n[0] // 2 + 2, 6, 6), n_steps=steps)
    return c


@pytest.mark.parametrize("kernel", [0, 4, 7])
@pytest.mark.parametrize("ranks", [2, 3])
def test_slab_engines_match_oracle(kernel, ranks):
    n, steps = (96, 20, 140), 6
    case = _case(n, steps)
    parts = slab.plan(n[0], ranks, x_cpml=(4, 3))
    run = slab.SlabEngines(slab.split(case, parts), parts, n_steps=steps,
                           options={"kernel": kernel})
    run.step(steps)
    run.sync()
    got = run.fields()
    run.close()
    orc = case.oracle()
    orc.run(steps)
    errs = [rel_l2(g, w) for g, w in zip(got, orc.e + orc.h)]
    assert max(errs) <= 1e-12, errs


def test_halo_copy_rejects_mismatched_lattices():
    from xfdtd_core_b200.engine import Engine, EngineError
    a = Engine(10, 8, 9, n_steps=2)
    b = Engine(10, 8, 10, n_steps=2)
    with pytest.raises(EngineError):
        a.halo_copy_from(0, b, 3, (1, 2))
    c = Engine(12, 8, 9, n_steps=2)
    with pytest.raises(EngineError):
        a.halo_copy_from(11, c, 3, (1,))  # plane 11 of a 10-cell lattice
    for e in (a, b, c):
        e.close()


@pytest.mark.parametrize("kernel", [0, 4, 7])
@pytest.mark.parametrize("ranks", [2, 3])
def test_slab_engines_with_tfsf_and_ade_match_oracle(kernel, ranks):
    n, steps = (96, 20, 140), 6
    case = KernelCase(n=n, seed=34, slabs=SLABS, field_scale=1e-3)
    case.tfsf = tfsf_source(n, (9, 4, 9), steps)
    # dispersive cells clear of the CPML layers, as in a scene (the host
    # builds the CPML coefficients from the dispersive nodes' own (ca, cb);
    # this synthetic case draws them independently)
    case.add_ade(kind=0, n_poles=2, n_mat=2, frac=0.2, margin=5)
    parts = slab.plan(n[0], ranks, x_cpml=(4, 3))
    run = slab.SlabEngines(slab.split(case, parts), parts, n_steps=steps,
                           options={"kernel": kernel})
    run.step(steps)
    run.sync()
    got = run.fields()
    run.close()
    orc = case.oracle()
    orc.run(steps)
    errs = [rel_l2(g, w) for g, w in zip(got, orc.e + orc.h)]
    assert max(errs) <= 1e-12, errs
