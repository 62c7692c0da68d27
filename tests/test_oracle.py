"""CPU checks of the oracle itself.  The reference ships no golden vectors
(parity unpinned), so these pin the restatement to properties the reference
algorithm must have: TFSF leaks no incident field into the scattered region,
mirror symmetry of a symmetric scene, an ADE medium without poles equals the
plain medium, the CPML absorbs, and the NF2FF nF-fold accumulation."""
import math

import numpy as np
import pytest

from oracle.reference_model import RefSimulation, EPSILON_0, MU_0, C_0
from xfdtd_core_b200 import scene as S


def _small_sphere(steps=160, **kw):
    base = dict(steps=steps, dl=0.35 / 20, radius=0.07, pml=6, tfsf_start=9, movie_interval=0)
    base.update(kw)
    return S.dielectric_sphere(**base)


def test_constants_match_reference():
    # include/xfdtd/common/constant.h:11-18
    assert EPSILON_0 == 8.854187817e-12
    assert MU_0 == 4 * math.pi * 1e-7
    assert abs(C_0 - 299792458.0) / 299792458.0 < 1e-9


def test_grid_matches_survey_sizes():
    r = RefSimulation(S.dielectric_sphere(steps=2))
    assert (r.nx, r.ny, r.nz) == (63, 63, 63)
    assert r.movies[0]["s"] == [8, 31, 8] and r.movies[0]["e"] == [55, 32, 55]


def test_tfsf_no_leakage_in_air():
    sc = _small_sphere(steps=200)
    sc.objects[1].material = S.air()
    r = RefSimulation(sc)
    s, e = r.tfsf["box_s"], r.tfsf["box_e"]
    tot, sca = 0.0, 0.0
    for _ in range(20):
        r.run(10)
        ex = r.e[0]
        tot = max(tot, np.abs(ex[s[0] + 1:e[0] - 1, s[1] + 1:e[1] - 1, s[2] + 1:e[2] - 1]).max())
        outside = np.abs(ex).copy()
        outside[s[0] - 1:e[0] + 1, s[1] - 1:e[1] + 2, s[2] - 1:e[2] + 2] = 0
        sca = max(sca, outside.max())
    assert tot > 0.5
    assert sca / tot < 1e-8


def test_mirror_symmetry_y():
    r = RefSimulation(_small_sphere(steps=120))
    r.run()
    ex = r.e[0]
    assert np.abs(ex).max() > 0
    assert np.abs(ex - ex[:, ::-1, :]).max() / np.abs(ex).max() < 1e-9


def test_ade_without_poles_equals_plain():
    def build(material):
        sc = S.dielectric_sphere(steps=80, dl=0.35 / 16, radius=0.06, pml=0, tfsf_start=4,
                                 movie_interval=0)
        sc.pmls = []
        sc.objects = [S.ObjectSpec("domain", sc.objects[0].shape, material)]
        return RefSimulation(sc)

    plain = build(S.Material("simple", 2.0, 1.0, 0.0, 0.0))
    ade = build(S.mlorentz(2.0, [0.0], [0.0], [1e20], [1e10], [1.0]))
    assert ade.ade is not None and ade.ade["kind"] == 0
    plain.run()
    ade.run()
    ref = max(np.linalg.norm(x) for x in plain.e)
    assert ref > 0
    for c in range(3):
        assert np.linalg.norm(ade.e[c] - plain.e[c]) / ref < 1e-12


def test_cpml_absorbs_dipole_pulse():
    def energy(pml):
        sc = S.dielectric_boxes(n=24 + 2 * pml, pml=pml, n_boxes=0, steps=300)
        if pml == 0:
            sc.pmls = []
        r = RefSimulation(sc)
        r.run()
        return sum(float(np.sum(x * x)) for x in r.e) * EPSILON_0 + \
            sum(float(np.sum(x * x)) for x in r.h) * MU_0

    assert energy(8) < 5e-3 * energy(0)


def test_nf2ff_accumulates_nf_times_per_step():
    def acc(freqs):
        sc = _small_sphere(steps=60, nf2ff_freqs=freqs, nf2ff_distance=4)
        r = RefSimulation(sc)
        r.run()
        return r.nf2ff_surface(0, 0, 0)

    one = acc([1e9])
    three = acc([1e9, 2e9, 3e9])
    assert np.abs(one).max() > 0
    np.testing.assert_allclose(three, 3 * one, rtol=1e-12, atol=1e-30)
