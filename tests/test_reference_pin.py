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
boxes with a lumped current source and graded CPML, and three ADE spheres
(Drude, modified Lorentz, Debye) under an oblique TFSF wave with a
frequency-domain NF2FF surface."""
import numpy as np
import pytest

from oracle.reference_model import RefSimulation
from tests import refpin
from tests.cases import rel_l2
from tests.scenes import boxes_small, dispersive_small, sphere_small
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
