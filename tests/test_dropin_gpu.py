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
"""
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
