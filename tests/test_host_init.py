"""The C++ host library's set-up (grid, painting, averaging, Yee
coefficients, lumped patch, CPML kappa, ADE overwrite), expanded back to the
reference's 18 coefficient arrays, against the oracle's restatement.  Runs
without a GPU (host set-up only)."""
import numpy as np
import pytest

from oracle.reference_model import RefSimulation
from tests.scenes import ALL
from xfdtd_core_b200.host import SceneRun

NAMES = ["cexe", "cexhy", "cexhz", "ceye", "ceyhz", "ceyhx", "ceze", "cezhx", "cezhy",
         "chxh", "chxey", "chxez", "chyh", "chyez", "chyex", "chzh", "chzex", "chzey"]


@pytest.mark.parametrize("name", sorted(ALL))
def test_coefficients_match_oracle(name):
    sc = ALL[name](steps=4)
    host = SceneRun(sc, engine=False)
    orc = RefSimulation(sc)
    assert host.n == (orc.nx, orc.ny, orc.nz)
    assert abs(host.dt - orc.dt) <= 1e-15 * orc.dt
    got = host.coefficients()
    want = []
    for c in range(3):
        want += [orc.ce[c], orc.ceh_a[c], orc.ceh_b[c]]
    for c in range(3):
        want += [orc.ch[c], orc.che_a[c], orc.che_b[c]]
    for nm, g, w in zip(NAMES, got, want):
        assert g.shape == w.shape, nm
        err = np.abs(g - w) / np.maximum(np.abs(w), 1e-300)
        assert err.max() <= 1e-13, (nm, float(err.max()), np.unravel_index(err.argmax(), err.shape))
