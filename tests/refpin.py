"""Runs a scene through the reference's own library (oracle/_ref/xfd_ref_driver,
built from the reference's unmodified sources by oracle/build_ref.py) and
reads back what it wrote: the six fields after the run, movie frames,
field-time monitors and frequency-domain far-field potentials."""
from __future__ import annotations

import glob
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "xfd_ref_driver")


def available() -> bool:
    return os.access(DRIVER, os.X_OK)


COEFFICIENTS = ("cexe", "cexhy", "cexhz", "ceye", "ceyhz", "ceyhx", "ceze", "cezhx", "cezhy",
                "chxh", "chxey", "chxez", "chyh", "chyez", "chyex", "chzh", "chzex", "chzey")


def run(scene, out_dir: str, steps: int | None = None, threads: int = 1,
        far_field: tuple | None = None, timeout: float = 1800,
        coefficients: bool = False) -> dict:
    """far_field = (n_theta, phi): processFarField over linspace(-pi, pi, n_theta).
    coefficients: also the 18 update-coefficient arrays as the run left them
    (out["coefficients"], in the order of COEFFICIENTS).  Voltage / current
    monitor series land in out["lines"], the network's S-parameters in
    out["s"] (keyed 10 j + i) and the radiated power in out["power"]."""
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "scene.txt")
    scene.write(path)
    cmd = [DRIVER, path, out_dir, "--threads", str(threads)]
    if steps is not None:
        cmd += ["--steps", str(steps)]
    if far_field is not None:
        cmd += ["--far-field", str(int(far_field[0])), repr(float(far_field[1]))]
    if coefficients:
        cmd += ["--coefficients"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference driver failed: {r.stderr[-2000:]}")
    out = {"fields": [np.load(os.path.join(out_dir, f"{c}.npy"))
                      for c in ("ex", "ey", "ez", "hx", "hy", "hz")]}
    for mv in scene.movies:
        frames = sorted(glob.glob(os.path.join(out_dir, mv.name, "*.npy")))
        out.setdefault("movies", {})[mv.name] = np.array([np.load(f) for f in frames])
    for ft in scene.field_times:
        out.setdefault("field_times", {})[ft.name] = np.load(
            os.path.join(out_dir, "field_time", f"{ft.name}.npy"))
    if coefficients:
        out["coefficients"] = [np.load(os.path.join(out_dir, "coef", f"{n}.npy"))
                               for n in COEFFICIENTS]
    for f in glob.glob(os.path.join(out_dir, "line", "*.npy")):
        out.setdefault("lines", {})[os.path.basename(f)[:-4]] = np.load(f)
    for f in glob.glob(os.path.join(out_dir, "network", "s*.npy")):
        out.setdefault("s", {})[int(os.path.basename(f)[1:-4])] = np.load(f)
    power = os.path.join(out_dir, "fd", "power.npy")
    if scene.nf2ff is not None and os.path.exists(power):
        out["power"] = np.load(power)
    if far_field is not None and scene.nf2ff is not None:
        ff = []
        for f in scene.nf2ff.freqs:
            tag = f"{f / 1e9:.2f}GHz"
            ff.append([np.load(os.path.join(out_dir, "fd", "ff", f"{tag}_{q}.npy"))
                       for q in ("a_theta", "f_phi", "a_phi", "f_theta")])
        out["far_field"] = np.array(ff)
    return out
