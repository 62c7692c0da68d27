"""The oracle pinned to the reference itself.

Scenes run through the reference's own library -- its unmodified src/**,
compiled into oracle/_ref by oracle/build_ref.py against the project's
xtensor subset -- and through the oracle restatement (oracle/reference_model.py
+ oracle/xfd_oracle.c) on the same scene text.  The fields after the run are
required to be identical bit for bit (both are FP64 without FMA contraction
and add the same terms in the same order); movie frames, field-time series
and far-field potentials (computed by the oracle from its own surface
currents) within 1e-12 relative L2.  Covered: the reference's
dielectric-sphere example (TFSF, PML, movie, field-time probe), dielectric
boxes with a lumped current source and graded CPML, three ADE spheres
(Drude, modified Lorentz, Debye) under an oblique TFSF wave with a
frequency-domain NF2FF surface, thin wires along all three axes with their
radiated power, every lumped element with voltage / current monitors, and
the reference's half-wave dipole example (thin-wire arms, voltage-source
port, one-port network).  The C++ host's set-up is pinned there too: its 18
update-coefficient arrays against the reference's."""
import numpy as np
import pytest

from oracle.reference_model import RefSimulation
from tests import refpin
from tests.cases import rel_l2
from oracle.reference_model import network_s_parameters
from tests.scenes import (boxes_small, dispersive_small, lumped_small, sphere_small,
                          wires_small)
from xfdtd_core_b200 import scene as S

pytestmark = pytest.mark.skipif(not refpin.available(),
                                reason="oracle/_ref not built (needs the reference sources)")
TOL = 1e-12
COMPONENTS = ("ex", "ey", "ez", "hx", "hy", "hz")


def _oracle(sc):
    orc = RefSimulation(sc)
    orc.run()
    return orc


@pytest.mark.parametrize("name,make", [("sphere", sphere_small), ("boxes", boxes_small),
                                       ("dispersive", dispersive_small)])
def test_fields_bit_equal_to_reference(tmp_path, name, make):
    sc = make(steps=150)
    ref = refpin.run(sc, str(tmp_path / name))
    orc = _oracle(sc)
    for c, got, want in zip(COMPONENTS, ref["fields"], orc.e + orc.h):
        assert got.shape == want.shape, c
        assert np.array_equal(got, want), (c, rel_l2(want, got))


def test_movie_and_field_time_match_reference(tmp_path):
    sc = sphere_small(steps=150)
    ref = refpin.run(sc, str(tmp_path))
    orc = _oracle(sc)
    mv = sc.movies[0].name
    want = np.array(orc.movie_frames[mv])
    assert ref["movies"][mv].shape == want.shape
    assert rel_l2(want, ref["movies"][mv]) <= TOL
    ft = sc.field_times[0].name
    got = ref["field_times"][ft]
    assert got.shape == orc.field_time_data[ft].shape
    np.testing.assert_array_equal(got[0], orc.field_time_data[ft][0])
    assert rel_l2(orc.field_time_data[ft][1], got[1]) <= TOL


def test_far_field_matches_reference(tmp_path):
    """NFFFTFrequencyDomain::processFarField of the reference (theta sweep
    over [-pi, pi] at phi = 30 deg) against the oracle's restatement of the
    potentials from its own surface currents."""
    sc = dispersive_small(steps=150)
    ref = refpin.run(sc, str(tmp_path), far_field=(37, np.pi / 6))
    orc = _oracle(sc)
    want = orc.far_field(np.linspace(-np.pi, np.pi, 37), np.pi / 6)
    assert ref["far_field"].shape == want.shape
    assert np.linalg.norm(ref["far_field"] - want) / np.linalg.norm(want) <= TOL


def test_dielectric_sphere_example_full_length(tmp_path):
    """The reference's dielectric-sphere example at its own size (63^3 with an
    8-cell PML, TFSF at 15, 2000 steps, an Ex XZ movie every 10 steps): the
    200 movie frames and the final fields of the reference and the oracle."""
    sc = S.dielectric_sphere(steps=2000)
    ref = refpin.run(sc, str(tmp_path), threads=4)
    orc = _oracle(sc)
    want = np.array(orc.movie_frames["movie_ex_xz"])
    assert ref["movies"]["movie_ex_xz"].shape == want.shape == (200, 47, 1, 47)
    assert rel_l2(want, ref["movies"]["movie_ex_xz"]) <= TOL
    for got, w in zip(ref["fields"], orc.e + orc.h):
        assert np.array_equal(got, w)


def _fields_equal(ref, orc):
    for c, got, want in zip(COMPONENTS, ref["fields"], orc.e + orc.h):
        assert got.shape == want.shape, c
        assert np.array_equal(got, want), (c, rel_l2(want, got))


def test_thin_wires_match_reference(tmp_path):
    """ThinWire along x, y and z (src/object/thin_wire.cpp): fields bit for
    bit, and the radiated power (outputRadiationPower) and far field of the
    NF2FF surface within 1e-12."""
    sc = wires_small(steps=150)
    ref = refpin.run(sc, str(tmp_path), far_field=(37, 0.5))
    orc = _oracle(sc)
    _fields_equal(ref, orc)
    np.testing.assert_array_equal(ref["power"][0], sc.nf2ff.freqs)
    want = orc.radiation_power()
    assert np.max(np.abs(ref["power"][1] - want) / np.abs(want)) <= TOL
    ff = orc.far_field(np.linspace(-np.pi, np.pi, 37), 0.5)
    assert np.linalg.norm(ref["far_field"] - ff) / np.linalg.norm(ff) <= TOL


def test_lumped_elements_and_monitors_match_reference(tmp_path):
    """Voltage and current sources, resistors, a capacitor and an inductor
    sharing nodes, and voltage / current monitors on them."""
    sc = lumped_small(steps=200)
    ref = refpin.run(sc, str(tmp_path))
    orc = _oracle(sc)
    _fields_equal(ref, orc)
    assert set(ref["lines"]) == set(orc.line_monitor_data)
    for name, got in ref["lines"].items():
        want = orc.line_monitor_data[name]
        np.testing.assert_array_equal(got[0], want[0])
        assert np.max(np.abs(got[1] - want[1])) <= TOL * np.max(np.abs(want[1])), name


def test_half_wave_dipole_example_matches_reference(tmp_path):
    """The reference's half-wave dipole example (test/src/examples/
    half_wave_dipole.cpp) at its own size, 600 of its 4000 steps: fields,
    the port's voltage and current, S11 over its 999 frequencies and the
    radiated power at 7 GHz."""
    sc = S.half_wave_dipole(steps=600)
    ref = refpin.run(sc, str(tmp_path))
    orc = _oracle(sc)
    _fields_equal(ref, orc)
    for name in ("v1", "c1"):
        want = orc.line_monitor_data[name][1]
        assert np.max(np.abs(ref["lines"][name][1] - want)) <= TOL * np.max(np.abs(want))
    s11 = network_s_parameters(orc, sc.network)[11]
    assert ref["s"][11].shape == s11.shape == (999,)
    assert np.linalg.norm(ref["s"][11] - s11) / np.linalg.norm(s11) <= TOL
    assert abs(ref["power"][1][0] - orc.radiation_power()[0]) <= TOL * abs(ref["power"][1][0])


@pytest.mark.parametrize("name,make", [("boxes", boxes_small), ("lumped", lumped_small),
                                       ("wires", wires_small), ("dispersive", dispersive_small)])
def test_host_coefficients_match_reference(tmp_path, name, make):
    """The C++ host's set-up (material classes x curl factors, lumped-element
    and thin-wire classes, H curl-term corrections; Simulation::
    coefficientArrays) against the reference's 18 FDTDUpdateCoefficient
    arrays after its init: within 1e-15 of each array's largest value."""
    from xfdtd_core_b200.host import SceneRun
    sc = make(steps=2)
    ref = refpin.run(sc, str(tmp_path), coefficients=True)
    run = SceneRun(sc, engine=False)
    for n, got, want in zip(refpin.COEFFICIENTS, run.coefficients(), ref["coefficients"]):
        assert got.shape == want.shape, n
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= 1e-15 * scale, (n, np.max(np.abs(got - want)))
    run.close()
