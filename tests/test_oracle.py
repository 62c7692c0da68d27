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


def test_grid_of_the_dielectric_sphere_example():
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


def _loop_far_field(orc, theta, phi_value, origin):
    """The reference's per-point loop (calculatePotential,
    src/nffft/nffft_fd_data_process.cpp:96-144) for one frequency, written out
    point by point in plain Python, for a single phi and an array of theta."""
    nf = orc.nf2ff
    freq = nf["freqs"][0]
    k0 = 2.0 * math.pi * freq / C_0
    out = np.zeros((4, len(theta)), dtype=np.complex128)
    for q, th in enumerate(theta):
        ct, st = math.cos(th), math.sin(th)
        cp, sp = math.cos(phi_value), math.sin(phi_value)
        t_theta = (ct * cp, ct * sp, -st)
        t_phi = (-sp, cp, 0.0)
        for row, (q0, tr) in enumerate([(0, t_theta), (2, t_phi), (0, t_phi), (2, t_theta)]):
            acc = 0j
            for face in range(6):
                if nf["tasks"][face] is None:
                    continue
                s, e = nf["tasks"][face]
                m = face // 2
                A, B = (m + 1) % 3, (m + 2) % 3
                a = orc.nf2ff_surface(0, face, q0)
                b = orc.nf2ff_surface(0, face, q0 + 1)
                for i in range(s[0], e[0]):
                    for j in range(s[1], e[1]):
                        for k in range(s[2], e[2]):
                            x = (i, j, k)
                            r = [(orc.e_node[d] if d == m else orc.h_node[d])[x[d]] - origin[d]
                                 for d in range(3)]
                            ds = orc.e_size[A][x[A]] * orc.e_size[B][x[B]]
                            arg = r[0] * st * cp + r[1] * st * sp + r[2] * ct
                            ph = complex(math.cos(k0 * arg), math.sin(k0 * arg))
                            v = a[i - s[0], j - s[1], k - s[2]] * tr[A] + \
                                b[i - s[0], j - s[1], k - s[2]] * tr[B]
                            acc += v * ph * ds
            out[row, q] = acc
    return out


def test_far_field_restatement_matches_loop_and_origin_shift():
    """The vectorised far-field restatement against the reference's point
    loop on a small scene, and the phase property of a moved origin: moving
    the origin by d multiplies every potential by exp(-i k d.rhat)."""
    sc = S.dispersive_spheres(n=24, pml=3, radius_cells=2, offsets_cells=((-4, 0), (2, 4), (2, -4)),
                              steps=30, tfsf_start=5, nf2ff_distance=4, n_freqs=2,
                              movie_interval=0)
    orc = RefSimulation(sc)
    orc.run()
    theta = np.linspace(0.1, math.pi - 0.1, 5)
    phi = math.pi / 6
    ff = orc.far_field(theta, phi)
    assert ff.shape == (2, 4, 5)
    assert np.abs(ff).max() > 0
    loop = _loop_far_field(orc, theta, phi, (0.0, 0.0, 0.0))
    assert np.linalg.norm(ff[0] - loop) <= 1e-12 * np.linalg.norm(loop)
    d = np.array([1.3e-3, -0.7e-3, 2.1e-3])
    moved = orc.far_field(theta, phi, origin=tuple(d))
    k0 = 2 * math.pi * orc.nf2ff["freqs"] / C_0
    rhat = np.stack([np.sin(theta) * math.cos(phi), np.sin(theta) * math.sin(phi), np.cos(theta)])
    shift = np.exp(-1j * k0[:, None] * (d @ rhat)[None, :])
    assert np.linalg.norm(moved - ff * shift[:, None, :]) <= 1e-11 * np.linalg.norm(ff)


def test_kernel_case_oracle_steps():
    """The kernel-level oracle (explicit arrays, no scene init) steps and
    changes the fields."""
    from tests.cases import KernelCase
    kc = KernelCase(seed=1)
    orc = kc.oracle()
    before = [f.copy() for f in orc.e]
    orc.run(2)
    assert orc.t == 2
    assert any(not np.array_equal(a, b) for a, b in zip(before, orc.e))


def _lumped_oracle():
    from tests.scenes import lumped_small
    sc = lumped_small(steps=4)
    orc = RefSimulation(sc)
    return sc, orc, {m["name"]: m["entries"] for m in orc.line_monitors}


def test_voltage_monitor_is_the_line_integral():
    """A uniform Ez = 3 V/m across the two-cell z-directed monitor reads
    V = -integral E.dl = -3 x 2 dl (the monitor's sign convention, ZP)."""
    sc, orc, entries = _lumped_oracle()
    v = sum(w * 3.0 for f, x, w in entries["v_vs"] if f == "EZ")
    assert abs(v - (-3.0 * 2 * sc.dl[0])) <= 1e-15


def test_current_monitor_closes_the_ampere_loop():
    """For Hx = -g y, Hy = g x (curl_z H = 2g everywhere) the current
    monitor's weighted H entries sum to 2 g times the area between its H rows
    and columns: the restated index ranges close the loop."""
    sc, orc, entries = _lumped_oracle()
    g = 2.5
    hn = orc.h_node
    total, xs, ys = 0.0, set(), set()
    for f, (i, j, k), w in entries["i_vs"]:
        if f == "HX":  # Hx(i, j, k) sits at y = h_node[1][j]
            total += w * (-g * hn[1][j])
            ys.add(float(hn[1][j]))
        elif f == "HY":  # Hy(i, j, k) sits at x = h_node[0][i]
            total += w * (g * hn[0][i])
            xs.add(float(hn[0][i]))
    area = (max(xs) - min(xs)) * (max(ys) - min(ys))
    assert area > 0
    assert abs(total - 2 * g * area) <= 1e-12 * 2 * g * area
