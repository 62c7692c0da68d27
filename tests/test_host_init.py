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


@pytest.mark.parametrize("name", ["sphere", "dispersive"])
def test_tfsf_tables_match_oracle(name):
    """The host's 1-D incident grid (every step) and projections equal the
    oracle's: the far-end Mur ABC of the 1-D grid turns last-ulp differences
    of the source into visible errors, so the tables must agree bit for bit
    wherever the source has not underflowed."""
    sc = ALL[name](steps=300)
    host = SceneRun(sc, engine=False)
    orc = RefSimulation(sc)
    t = orc.tfsf
    size = [t["box_e"][a] - t["box_s"][a] for a in range(3)]
    e_inc, h_inc, p_int, p_half = host.tfsf_tables(size)
    assert e_inc.shape == t["e_inc"].shape
    scale = np.abs(t["e_inc"]).max()
    assert np.abs(e_inc - t["e_inc"]).max() <= 1e-30 * scale
    assert np.abs(h_inc - t["h_inc"]).max() <= 1e-30 * scale
    for a in range(3):
        assert np.array_equal(p_int[a], t["p_int"][a])
        assert np.array_equal(p_half[a], t["p_half"][a])


def test_batched_workload_parameters():
    """The batched workload's 96 scenes: sizes log-uniform in [64, 224]
    (mean N^3 about 2.9 M cells), reproducible from the seed."""
    from xfdtd_core_b200 import scene as S
    p = S.batched_sphere_params()
    assert len(p) == 96 and p == S.batched_sphere_params()
    n = np.array([q["n"] for q in p])
    assert n.min() >= 64 and n.max() <= 224
    assert 2.5e6 < float((n.astype(float) ** 3).mean()) < 3.3e6
    for q in p:
        assert 0.1 * q["n"] <= q["radius_cells"] <= 0.3 * q["n"]
        assert 2 <= q["eps_r"] <= 10 and 0 <= q["theta"] <= np.pi


def test_random_angle_tfsf_tables_match_oracle():
    """A batched-workload scene (random theta, phi, psi): the host's TFSF
    tables equal the oracle's, as for the fixed-angle scenes."""
    from xfdtd_core_b200 import scene as S
    sc = S.batched_sphere(n=40, radius_cells=8.0, eps_r=5.0, theta=2.2, phi=4.1, psi=0.7,
                          pml=6, tfsf_start=9, steps=200)
    host = SceneRun(sc, engine=False)
    orc = RefSimulation(sc)
    t = orc.tfsf
    size = [t["box_e"][a] - t["box_s"][a] for a in range(3)]
    e_inc, h_inc, p_int, p_half = host.tfsf_tables(size)
    scale = np.abs(t["e_inc"]).max()
    assert np.abs(e_inc - t["e_inc"]).max() <= 1e-30 * scale
    assert np.abs(h_inc - t["h_inc"]).max() <= 1e-30 * scale
    for a in range(3):
        assert np.array_equal(p_int[a], t["p_int"][a])
        assert np.array_equal(p_half[a], t["p_half"][a])


def test_scene_text_lines_for_lumped_network_and_pec_planes():
    """The scene lines of the lumped elements, PEC planes and the network
    round-trip through the host parser (host set-up only)."""
    from tests.scenes import lumped_small, microstrip_small
    for sc in (lumped_small(steps=4), microstrip_small(steps=4)):
        text = sc.to_text()
        for kw in ("voltage_source", "current_monitor", "voltage_monitor"):
            assert kw in text
        host = SceneRun(sc, engine=False)
        assert host.n[0] > 0
        host.close()
    text = microstrip_small(steps=4).to_text()
    assert "pec_plane microstrip_0" in text and "pec_plane ground_0" in text
    assert "network 40 " in text and "port 1 1 " in text
    text = lumped_small(steps=4).to_text()
    for kw in ("resistor r1", "capacitor c1", "inductor l1"):
        assert kw in text


def test_pec_plane_coefficients_are_pec_on_the_plane():
    """On the microstrip's ground plane (z = 0) the tangential E components
    take the PEC sigma_e: ca ~ -1, cb ~ 0; Ez there is untouched."""
    from tests.scenes import microstrip_small
    host = SceneRun(microstrip_small(steps=4), engine=False)
    co = host.coefficients()
    orc = RefSimulation(microstrip_small(steps=4))
    k0 = orc.grid_box(microstrip_small(steps=4).pec_planes[1].shape)[0][2]
    cexe, ceye = co[0], co[3]
    i0, j0, _ = orc.grid_box(microstrip_small(steps=4).pec_planes[1].shape)[0]
    assert cexe[i0 + 1, j0 + 1, k0] < -0.99 and ceye[i0 + 1, j0 + 1, k0] < -0.99
    assert cexe[i0 + 1, j0 + 1, k0 + 1] > 0.9
    host.close()
