"""The reference's own example programs, compiled unmodified against this
library's drop-in headers (tests/examples_build.py), run on the GPU and
checked against the oracle on the same scene: what each program writes --
far-field potentials, time-domain far-field series, port voltage and
current, S11, radiated power -- within 1e-12 relative L2 (FP64).

* dielectric_sphere_scatter.cpp: 133^3 with an 8-cell PML, TFSF at 15, a
  1 GHz frequency-domain and a time-domain NF2FF surface 11 cells in, 4800
  steps; processFarField over the xz and yz planes and the time-domain
  w/u series.
* half_wave_dipole.cpp: two ThinWire arms fed by a 50-ohm voltage source,
  a one-port network over 999 frequencies, a 7 GHz NF2FF surface, 4000
  steps; V/I monitors, S11, outputRadiationPower and three far-field cuts.
* dielectric_cube_scatter.cpp: 72^3, an eps_r = 5 cube under an oblique
  TFSF wave (theta = 45 deg, phi = 30 deg), 2000 steps; three far-field cuts
  at 1 GHz.
* dispersive_sphere_scatter/drude_sphere_scatter.cpp: the 63^3 sphere as a
  Drude medium (DrudeMedium, ADE), 1000 steps; two Ex movies (every 10th
  step, written by the MovieMonitors), three far-field cuts and
  relativePermittivity.
* microstrip_line.cpp: the voltage and current monitors and the one-port
  network's S11 over 500 frequencies.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from oracle.reference_model import RefSimulation, network_s_parameters
from tests import examples_build as X
from xfdtd_core_b200 import scene as S

pytestmark = pytest.mark.gpu
TOL = 1e-12
POT = ("a_theta", "f_phi", "a_phi", "f_theta")


def _run_example(name, cwd):
    exe = os.path.join(X.OUT, name)
    if not os.access(exe, os.X_OK):
        pytest.fail(f"{exe} is not built (tests/examples_build.py)")
    r = subprocess.run([exe], cwd=cwd, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr[-3000:]


def _rel(got, want):
    return float(np.linalg.norm(np.asarray(got) - want) / np.linalg.norm(want))


def _far(directory, sub, freq):
    tag = f"{freq / 1e9:.2f}GHz"
    return np.array([np.load(os.path.join(directory, sub, f"{tag}_{q}.npy")) for q in POT])


def test_dielectric_sphere_example_matches_oracle(tmp_path):
    _run_example("dielectric_sphere_scatter", str(tmp_path))
    out = tmp_path / "tmp" / "data" / "dielectric_sphere_scatter"
    sc = S.dielectric_sphere(steps=4800, dl=3e-3, movie_interval=0, nf2ff_freqs=[1e9],
                             nf2ff_distance=11)
    sc.nf2ff_td = S.NF2FFTDSpec((11, 11, 11), -np.pi, 0.0)
    orc = RefSimulation(sc)
    assert (orc.nx, orc.ny, orc.nz) == (133, 133, 133)
    orc.run()
    sweep = np.linspace(-np.pi, np.pi, 360)
    for sub, phi in (("xz", 0.0), ("yz", np.pi * 0.5)):
        got = _far(out / "fd", sub, 1e9)
        want = orc.far_field(sweep, phi)[0]
        assert got.shape == want.shape == (4, 360)
        assert _rel(got, want) <= TOL, (sub, _rel(got, want))
    td = orc.nf2ff_td_far_field()
    for key in ("w_theta", "w_phi", "u_theta", "u_phi"):
        got = np.load(out / "td" / f"{key}.npy")
        assert got.shape == td[key].shape, key
        assert _rel(got, td[key]) <= TOL, (key, _rel(got, td[key]))
    t = np.load(out / "time.npy")
    assert t.shape == (4800,)


def test_half_wave_dipole_example_matches_oracle(tmp_path):
    _run_example("half_wave_dipole", str(tmp_path))
    sc = S.half_wave_dipole(steps=4000)
    orc = RefSimulation(sc)
    orc.run()
    mon = tmp_path / "data" / "half_wave_dipole"
    for name in ("v1", "c1"):
        got = np.load(mon / f"{name}.npy")
        want = orc.line_monitor_data[name]
        np.testing.assert_array_equal(got[0], want[0])
        assert _rel(got[1], want[1]) <= TOL, name
    out = tmp_path / "tmp" / "data" / "half_wave_dipole"
    s11 = network_s_parameters(orc, sc.network)[11]
    got = np.load(out / "s11.npy")
    assert got.shape == s11.shape == (999,)
    assert _rel(got, s11) <= TOL
    np.testing.assert_array_equal(np.load(out / "frequencies.npy"), sc.network.frequencies)
    power = np.load(out / "power.npy")
    assert power.shape == (2, 1) and power[0, 0] == 7e9
    want_p = orc.radiation_power()[0]
    assert abs(power[1, 0] - want_p) <= TOL * abs(want_p)
    sweep = np.linspace(-np.pi, np.pi, 360)
    cuts = {"xy": (np.pi * 0.5, sweep), "xz": (sweep, 0.0), "yz": (sweep, np.pi * 0.5)}
    for sub, (theta, phi) in cuts.items():
        got = _far(out, sub, 7e9)
        want = orc.far_field(theta, phi)[0]
        assert _rel(got, want) <= TOL, (sub, _rel(got, want))


def test_dielectric_cube_example_matches_oracle(tmp_path):
    _run_example("dielectric_cube_scatter", str(tmp_path))
    out = tmp_path / "tmp" / "data" / "dielectric_cube_scatter" / "fd"
    dl, half = 5e-3, 80e-3
    sc = S.Scene(dl=(dl, dl, dl), cfl=0.9, steps=2000, name="dielectric_cube")
    sc.objects.append(S.ObjectSpec("domain", S.cube((-half - 10 * dl,) * 3,
                                                    (2 * half + 20 * dl,) * 3), S.air()))
    sc.objects.append(S.ObjectSpec("dielectric_cube", S.cube((-half,) * 3, (2 * half,) * 3),
                                   S.Material("simple", 5.0, 1.0, 0.0, 0.0)))
    tau = dl * 20 / 6e8
    sc.tfsf = S.TFSFSpec(15, 15, 15, math.pi * 0.25, math.pi / 6.0, 0.0,
                         S.Waveform("gaussian", tau, 4.5 * tau))
    sc.nf2ff = S.NF2FFSpec((13, 13, 13), [1e9])
    sc.pmls = S.pml_all(10)
    orc = RefSimulation(sc)
    assert (orc.nx, orc.ny, orc.nz) == (72, 72, 72)
    orc.run()
    sweep = np.linspace(-np.pi, np.pi, 360)
    cuts = {"xy": (np.pi * 0.5, sweep), "xz": (sweep, 0.0), "yz": (sweep, np.pi * 0.5)}
    for sub, (theta, phi) in cuts.items():
        got = _far(out, sub, 1e9)
        want = orc.far_field(theta, phi)[0]
        assert _rel(got, want) <= TOL, (sub, _rel(got, want))


def test_drude_sphere_example_matches_oracle(tmp_path):
    import glob
    _run_example("drude_sphere_scatter", str(tmp_path))
    out = tmp_path / "data" / "dispersive_material_scatter" / "drude_medium"
    sc = S.dielectric_sphere(steps=1000, movie_interval=10, nf2ff_freqs=[1e9], nf2ff_distance=11)
    sc.objects[1].material = S.drude(4.0, [math.pi * 1e9], [math.pi * 1.2e9])
    half, dl = 0.175, 7.5e-3
    sc.movies.append(S.MovieSpec("movie_ex_yz", "EX",
                                 S.cube((0.0, -half, -half), (dl, 2 * half, 2 * half)), 10))
    orc = RefSimulation(sc)
    orc.run()
    for name in ("movie_ex_xz", "movie_ex_yz"):
        files = sorted(glob.glob(str(out / name / "*.npy")))
        want = np.array(orc.movie_frames[name])
        assert len(files) == len(want) == 100, name
        assert os.path.basename(files[1]) == "00010.npy"
        got = np.array([np.load(f) for f in files])
        assert got.shape == want.shape
        assert _rel(got, want) <= TOL, (name, _rel(got, want))
    sweep = np.linspace(-np.pi, np.pi, 360)
    cuts = {"xy": (np.pi * 0.5, sweep), "xz": (sweep, 0.0), "yz": (sweep, np.pi * 0.5)}
    for sub, (theta, phi) in cuts.items():
        got = _far(out / "fd", sub, 1e9)
        want = orc.far_field(theta, phi)[0]
        assert _rel(got, want) <= TOL, (sub, _rel(got, want))
    eps = np.load(out / "relative_permittivity.npy")
    f = np.linspace(1e7, 5e9, 100)
    w = 2 * np.pi * f
    want = 4.0 + (math.pi * 1e9) ** 2 / ((1j * w) ** 2 + math.pi * 1.2e9 * 1j * w)
    assert eps.shape == (2, 100)
    np.testing.assert_allclose(eps[0].real, f, rtol=1e-15)
    np.testing.assert_allclose(eps[1], want, rtol=1e-13)


def test_microstrip_line_example_matches_oracle(tmp_path):
    _run_example("microstrip_line", str(tmp_path))
    out = tmp_path / "data" / "microstrip_line"
    sc = S.microstrip_line()
    orc = RefSimulation(sc)
    orc.run()
    for name in ("v1", "c1"):
        got = np.load(out / f"{name}.npy")
        want = orc.line_monitor_data[name]
        np.testing.assert_array_equal(got[0], want[0])
        assert _rel(got[1], want[1]) <= TOL, name
    s11 = network_s_parameters(orc, sc.network)[11]
    got = np.load(out / "s11.npy")
    assert got.shape == s11.shape == (500,)
    assert _rel(got, s11) <= TOL
