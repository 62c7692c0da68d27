"""Scene descriptions for the XFDTD 3-D hot path.

A :class:`Scene` is the data a user program hands to ``xfdtd::Simulation``
(objects, boundaries, sources, monitors, NF2FF, step count).  It mirrors the
reference's user-facing API one to one:

* ``Object(name, Cube|Sphere, Material)``            include/xfdtd/object/object.h:28-29
* ``ElectroMagneticProperty(eps_r, mu_r, s_e, s_m)`` src/material/material.cpp:11-26
* ``DrudeMedium / DebyeMedium / MLorentzMaterial``   include/xfdtd/material/dispersive_material.h:71-122
* ``PML(thickness, dir, order, sigma_ratio, alpha_min, alpha_max, kappa_max)``
                                                       include/xfdtd/boundary/pml.h:19-21
* ``TFSF3D(x, y, z, theta, phi, psi, waveform)``      include/xfdtd/waveform_source/tfsf_3d.h:10-11
* ``CurrentSource(name, cube, dir, R, waveform)``     include/xfdtd/object/lumped_element/current_source.h:11-14
* ``VoltageSource(name, cube, dir, R, waveform)``     include/xfdtd/object/lumped_element/voltage_source.h:15-18
* ``Network(ports, freqs) / Port(i, src, z, c, v)``   include/xfdtd/network/{network,port}.h
* ``PecPlane(name, cube)``                            include/xfdtd/object/lumped_element/pec_plane.h:10-12
* ``ThinWire(name, Cylinder(center, r, h, axis))``   include/xfdtd/object/thin_wire.h:14-16
* ``Resistor / Capacitor / Inductor(name, cube, xyz, value)``
                                                       include/xfdtd/object/lumped_element/{resistor,capacitor,inductor}.h:9-12
* ``MovieMonitor(FieldMonitor(cube, field), k)``      include/xfdtd/monitor/movie_monitor.h:13-15
* ``NFFFTFrequencyDomain(dx, dy, dz, freqs)``         include/xfdtd/nffft/nffft_frequency_domain.h:19-45
* ``Waveform::gaussian / cosineModulatedGaussian``    src/waveform/waveform.cpp:80-96

``Scene.to_text()`` serialises the scene into the line format that the C++
host library (``xfdtd_scene_open``) parses into exactly those API calls, with
every float printed as a round-trip ``repr`` so both sides see identical
doubles.  The workload builders at the bottom define the five benchmark
scenes (dielectric sphere, dielectric boxes, dispersive spheres) with a size
knob so that the same geometry rule gives small parity cases.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

Vec3 = Tuple[float, float, float]

DIRECTIONS = ("XN", "XP", "YN", "YP", "ZN", "ZP")
FIELDS = ("EX", "EY", "EZ", "HX", "HY", "HZ")


def _f(x: float) -> str:
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return repr(float(x))


@dataclass
class Waveform:
    """``Waveform::gaussian(tau, t0)`` or ``cosineModulatedGaussian(tau, t0, f)``."""

    kind: str  # "gaussian" | "cosgauss"
    tau: float
    t0: float
    freq: float = 0.0
    amplitude: float = 1.0

    def text(self) -> str:
        if self.kind == "gaussian":
            return f"gaussian {_f(self.tau)} {_f(self.t0)} {_f(self.amplitude)}"
        if self.kind == "cosgauss":
            return (f"cosgauss {_f(self.tau)} {_f(self.t0)} {_f(self.freq)} "
                    f"{_f(self.amplitude)}")
        raise ValueError(self.kind)

    def __call__(self, t):
        """Samples the waveform like ``Waveform::init`` (waveform.cpp:28-34),
        element by element with the C library's exp/pow/cos (the functions
        std::exp/std::pow/std::cos call), not numpy's vectorised ones, whose
        last-ulp results differ."""
        t = np.asarray(t, dtype=np.float64)
        out = np.empty(t.shape)
        flat, res = t.ravel(), out.ravel()
        for q, tv in enumerate(flat.tolist()):
            g = math.exp(-math.pow((tv - self.t0) / self.tau, 2))
            if self.kind == "gaussian":
                v = g
            else:
                v = g * math.cos(2 * math.pi * self.freq * (tv - self.t0))
            res[q] = self.amplitude * v
        return out


@dataclass
class Material:
    """A simple (eps_r, mu_r, sigma_e, sigma_m) medium or a linear dispersive one.

    ``kind`` is "simple", "drude", "debye" or "mlorentz".  Dispersive media
    carry ``eps_inf`` and per-pole parameter lists; their em-property is air
    (``ElectroMagneticProperty::air()``), as the reference factories build them.
    """

    kind: str = "simple"
    eps_r: float = 1.0
    mu_r: float = 1.0
    sigma_e: float = 0.0
    sigma_m: float = 0.0
    eps_inf: float = 1.0
    # drude: omega_p, gamma; debye: eps_static, tau; mlorentz: a0, a1, b0, b1, b2
    poles: List[Tuple[float, ...]] = field(default_factory=list)

    def text(self) -> str:
        if self.kind == "simple":
            return (f"simple {_f(self.eps_r)} {_f(self.mu_r)} {_f(self.sigma_e)} "
                    f"{_f(self.sigma_m)}")
        body = " ".join(" ".join(_f(v) for v in p) for p in self.poles)
        return f"{self.kind} {_f(self.eps_inf)} {len(self.poles)} {body}"

    @property
    def dispersive(self) -> bool:
        return self.kind != "simple"


def air() -> Material:
    return Material("simple", 1.0, 1.0, 0.0, 0.0)


def drude(eps_inf: float, omega_p: Sequence[float], gamma: Sequence[float]) -> Material:
    return Material("drude", eps_inf=eps_inf,
                    poles=[(float(w), float(g)) for w, g in zip(omega_p, gamma)])


def debye(eps_inf: float, eps_static: Sequence[float], tau: Sequence[float]) -> Material:
    return Material("debye", eps_inf=eps_inf,
                    poles=[(float(e), float(t)) for e, t in zip(eps_static, tau)])


def mlorentz(eps_inf: float, a0, a1, b0, b1, b2) -> Material:
    return Material("mlorentz", eps_inf=eps_inf,
                    poles=[tuple(float(v) for v in p) for p in zip(a0, a1, b0, b1, b2)])


@dataclass
class Shape:
    kind: str  # "cube" | "sphere" | "cylinder"
    origin: Vec3  # cube origin, sphere or cylinder centre
    size: Vec3 = (0.0, 0.0, 0.0)  # cube size
    radius: float = 0.0
    height: float = 0.0  # cylinder length along its axis
    axis: int = 2  # cylinder axis: 0, 1, 2 for x, y, z

    def text(self) -> str:
        if self.kind == "cube":
            return "cube " + " ".join(_f(v) for v in (*self.origin, *self.size))
        if self.kind == "cylinder":
            return ("cylinder " + " ".join(_f(v) for v in (*self.origin, self.radius, self.height))
                    + " " + "XYZ"[self.axis])
        return "sphere " + " ".join(_f(v) for v in (*self.origin, self.radius))


def cube(origin: Vec3, size: Vec3) -> Shape:
    return Shape("cube", tuple(map(float, origin)), tuple(map(float, size)))


def sphere(center: Vec3, radius: float) -> Shape:
    return Shape("sphere", tuple(map(float, center)), radius=float(radius))


def cylinder(center: Vec3, radius: float, height: float, axis: int) -> Shape:
    """``Cylinder(center, radius, height, Axis)`` (src/shape/cylinder.cpp:13-26)."""
    return Shape("cylinder", tuple(map(float, center)), radius=float(radius),
                 height=float(height), axis=int(axis))


@dataclass
class ObjectSpec:
    name: str
    shape: Shape
    material: Material

    def text(self) -> str:
        return f"object {self.name} {self.shape.text()} {self.material.text()}"


@dataclass
class VoxelSpec:
    """A block of per-voxel relative permittivities (xfdtd::VoxelObject): the
    cube (origin, size) divided into eps_r.shape voxels; a cell whose centre
    lies in the cube is painted (in object order, like any object) with the
    eps_r of the voxel holding its centre and the common mu_r, sigma_e."""
    name: str
    origin: Vec3
    size: Vec3
    eps_r: np.ndarray
    mu_r: float = 1.0
    sigma_e: float = 0.0

    @property
    def shape(self) -> Shape:
        return cube(self.origin, self.size)

    @property
    def material(self) -> Material:
        return Material("simple", float(np.mean(self.eps_r)), self.mu_r, self.sigma_e, 0.0)

    def voxel_index(self, a: int, centre: np.ndarray) -> np.ndarray:
        """Voxel index along axis a of cell centres (VoxelObject's rule)."""
        n = self.eps_r.shape[a]
        w = self.size[a] / n
        q = np.floor((centre - self.origin[a]) / w).astype(np.int64)
        return np.clip(q, 0, n - 1)

    def text(self) -> str:
        e = np.asarray(self.eps_r, dtype=np.float64)
        return (f"voxels {self.name} " + " ".join(_f(v) for v in (*self.origin, *self.size)) +
                f" {e.shape[0]} {e.shape[1]} {e.shape[2]} {_f(self.mu_r)} {_f(self.sigma_e)} " +
                " ".join(repr(float(v)) for v in e.ravel()))


@dataclass
class CurrentSourceSpec:
    name: str
    shape: Shape  # a Cube
    direction: str
    resistance: float
    waveform: Waveform
    kind: str = "current"  # "current" | "voltage"

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return (f"{self.kind}_source {self.name} " +
                " ".join(_f(v) for v in (*o, *s)) +
                f" {self.direction} {_f(self.resistance)} {self.waveform.text()}")


@dataclass
class VoltageSourceSpec(CurrentSourceSpec):
    kind: str = "voltage"


@dataclass
class PortSpec:
    """``Port(index, is_source, impedance, current_monitor, voltage_monitor)``
    with the monitors named."""
    index: int
    is_source: bool
    impedance: complex
    current: str
    voltage: str

    def text(self) -> str:
        z = complex(self.impedance)
        return (f"port {self.index} {int(bool(self.is_source))} {_f(z.real)} {_f(z.imag)} "
                f"{self.current} {self.voltage}")


@dataclass
class NetworkSpec:
    """``Network(ports, frequencies, output_dir)``."""
    frequencies: List[float]
    ports: List[PortSpec] = field(default_factory=list)

    def text(self) -> str:
        return "\n".join([f"network {len(self.frequencies)} " +
                          " ".join(_f(float(f)) for f in self.frequencies)] +
                         [p.text() for p in self.ports])


@dataclass
class PecPlaneSpec:
    """``PecPlane(name, cube)``: a Cube flat on one axis."""
    name: str
    shape: Shape

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return f"pec_plane {self.name} " + " ".join(_f(v) for v in (*o, *s))


@dataclass
class ThinWireSpec:
    """``ThinWire(name, Cylinder)`` (src/object/thin_wire.cpp): an air object
    whose E along the wire is held at zero and whose neighbouring H
    coefficients take the thin-wire factor."""
    name: str
    shape: Shape  # a cylinder

    def text(self) -> str:
        sh = self.shape
        return (f"thin_wire {self.name} " + " ".join(_f(v) for v in (*sh.origin, sh.radius,
                                                                      sh.height))
                + " " + "XYZ"[sh.axis])


@dataclass
class LumpedSpec:
    """Resistor, Capacitor or Inductor (kind "resistor" | "capacitor" |
    "inductor") on a Cube of E nodes along `axis` ("X" | "Y" | "Z")."""
    kind: str
    name: str
    shape: Shape  # a Cube
    axis: str
    value: float

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return (f"{self.kind} {self.name} " + " ".join(_f(v) for v in (*o, *s)) +
                f" {self.axis} {_f(self.value)}")


@dataclass
class PMLSpec:
    thickness: int
    direction: str
    order: int = 4
    sigma_ratio: float = 1.0
    alpha_min: float = 0.0
    alpha_max: float = 0.05
    kappa_max: float = 10.0

    def text(self) -> str:
        return (f"pml {self.thickness} {self.direction} {self.order} "
                f"{_f(self.sigma_ratio)} {_f(self.alpha_min)} {_f(self.alpha_max)} "
                f"{_f(self.kappa_max)}")


@dataclass
class TFSFSpec:
    x: int
    y: int
    z: int
    theta: float
    phi: float
    psi: float
    waveform: Waveform

    def text(self) -> str:
        return (f"tfsf3d {self.x} {self.y} {self.z} {_f(self.theta)} {_f(self.phi)} "
                f"{_f(self.psi)} {self.waveform.text()}")


@dataclass
class MovieSpec:
    name: str
    field: str
    shape: Shape  # Cube
    interval: int

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return (f"movie {self.name} {self.field} " +
                " ".join(_f(v) for v in (*o, *s)) + f" {self.interval}")


@dataclass
class FieldTimeSpec:
    """FieldTimeMonitor(name, cube, dir, field): the field at the last node of
    the cube's node box, every step (src/monitor/field_time_monitor.cpp:81-95)."""
    name: str
    field: str
    shape: Shape  # Cube

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return (f"field_time {self.name} {self.field} " +
                " ".join(_f(v) for v in (*o, *s)))


@dataclass
class NF2FFSpec:
    distance: Tuple[int, int, int]
    freqs: Sequence[float]

    def text(self) -> str:
        d = self.distance
        return (f"nf2ff_fd {d[0]} {d[1]} {d[2]} {len(self.freqs)} " +
                " ".join(_f(f) for f in self.freqs))


@dataclass
class LineMonitorSpec:
    """VoltageMonitor / CurrentMonitor(name, cube, direction): `kind` is
    "voltage" or "current"."""
    kind: str
    name: str
    shape: Shape  # Cube
    direction: str

    def text(self) -> str:
        o, s = self.shape.origin, self.shape.size
        return (f"{self.kind}_monitor {self.name} " + " ".join(_f(v) for v in (*o, *s)) +
                f" {self.direction}")


@dataclass
class NF2FFTDSpec:
    """NFFFTTimeDomain(distance_x, distance_y, distance_z, theta, phi)."""
    distance: Tuple[int, int, int]
    theta: float
    phi: float

    def text(self) -> str:
        d = self.distance
        return f"nf2ff_td {d[0]} {d[1]} {d[2]} {_f(self.theta)} {_f(self.phi)}"


@dataclass
class Scene:
    """Everything a reference user program passes to ``xfdtd::Simulation``."""

    dl: Vec3
    cfl: float
    steps: int
    objects: List[ObjectSpec] = field(default_factory=list)
    thin_wires: List[ThinWireSpec] = field(default_factory=list)
    current_sources: List[CurrentSourceSpec] = field(default_factory=list)
    lumped_elements: List[LumpedSpec] = field(default_factory=list)
    pec_planes: List[PecPlaneSpec] = field(default_factory=list)
    pmls: List[PMLSpec] = field(default_factory=list)
    tfsf: Optional[TFSFSpec] = None
    movies: List[MovieSpec] = field(default_factory=list)
    field_times: List[FieldTimeSpec] = field(default_factory=list)
    line_monitors: List[LineMonitorSpec] = field(default_factory=list)
    nf2ff: Optional[NF2FFSpec] = None
    nf2ff_td: Optional[NF2FFTDSpec] = None
    network: Optional[NetworkSpec] = None
    name: str = "scene"

    def to_text(self) -> str:
        lines = ["xfdtd-scene 1", f"name {self.name}",
                 "grid " + " ".join(_f(v) for v in self.dl) + f" {_f(self.cfl)}",
                 f"steps {self.steps}"]
        lines += [o.text() for o in self.objects]
        lines += [w.text() for w in self.thin_wires]
        lines += [c.text() for c in self.current_sources]
        lines += [c.text() for c in self.lumped_elements]
        lines += [c.text() for c in self.pec_planes]
        lines += [p.text() for p in self.pmls]
        if self.tfsf is not None:
            lines.append(self.tfsf.text())
        lines += [m.text() for m in self.movies]
        lines += [m.text() for m in self.field_times]
        lines += [m.text() for m in self.line_monitors]
        if self.nf2ff is not None:
            lines.append(self.nf2ff.text())
        if self.nf2ff_td is not None:
            lines.append(self.nf2ff_td.text())
        if self.network is not None:
            lines.append(self.network.text())
        return "\n".join(lines) + "\n"

    def write(self, path: str) -> str:
        with open(path, "w") as fh:
            fh.write(self.to_text())
        return path


def pml_all(thickness: int, **kw) -> List[PMLSpec]:
    return [PMLSpec(thickness, d, **kw) for d in DIRECTIONS]


# ---------------------------------------------------------------------------
# Workloads.  Each keeps its geometry rule for every size so that the small
# variants used by the parity tests exercise the same code paths.
# ---------------------------------------------------------------------------

def dielectric_sphere(steps: int = 2000, dl: float = 7.5e-3, half: float = 0.175,
                      radius: float = 0.1, pml: int = 8, tfsf_start: int = 15,
                      movie_interval: int = 10, nf2ff_freqs: Sequence[float] = (),
                      nf2ff_distance: int = 11) -> Scene:
    """Plain FP64 dielectric-sphere scatter (the reference's
    test/src/examples/dielectric_sphere_scatter.cpp:26-129 at dl=7.5e-3):
    0.35 m air cube, 8-cell PML, sphere r=0.1 eps_r=3 mu_r=2, TFSF3D at index
    15 with a Gaussian (tau = 20*dl/6e8, t0 = 4.5 tau), CFL 0.9, an Ex XZ-plane
    movie every 10 steps."""
    tau = dl * 20 / 6e8
    s = Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps, name="dielectric_sphere")
    s.objects.append(ObjectSpec("domain", cube((-half,) * 3, (2 * half,) * 3), air()))
    s.objects.append(ObjectSpec("dielectric_sphere", sphere((0, 0, 0), radius),
                                Material("simple", 3.0, 2.0, 0.0, 0.0)))
    s.pmls = pml_all(pml)
    s.tfsf = TFSFSpec(tfsf_start, tfsf_start, tfsf_start, 0.0, 0.0, 0.0,
                      Waveform("gaussian", tau, 4.5 * tau))
    if movie_interval:
        s.movies.append(MovieSpec("movie_ex_xz", "EX",
                                  cube((-half, 0.0, -half), (2 * half, dl, 2 * half)),
                                  movie_interval))
        # the example's scattered-field probe (dielectric_sphere_scatter.cpp:85-90)
        s.field_times.append(FieldTimeSpec("ex_point", "EX",
                                           cube((0.0, -half + 3 * dl, 0.0), (dl, dl, dl))))
    if nf2ff_freqs:
        s.nf2ff = NF2FFSpec((nf2ff_distance,) * 3, list(nf2ff_freqs))
    return s


def half_wave_dipole(steps: int = 4000, dl: float = 2.5e-4, arm_cells: int = 39,
                     pad_cells: int = 10, pml: int = 8, nf2ff_distance: int = 13,
                     nf2ff_freqs: Sequence[float] = (7e9,), network: bool = True) -> Scene:
    """The reference's half-wave dipole (test/src/examples/half_wave_dipole.cpp:
    20-99): two z-directed ThinWire arms of radius 5e-5 and length arm_cells dl
    either side of a two-cell 50-ohm voltage source gap (Gaussian, tau =
    30 dl / 6e8), an air domain pad_cells beyond the arms on every side, an
    8-cell PML, a voltage / current monitor port on the gap with a one-port
    network over 20 MHz .. 20 GHz, and a frequency-domain NF2FF surface 13
    cells in."""
    reach = (arm_cells + 1) * dl  # the arms end at z = +-(arm_cells + 1) dl
    s = Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps, name="half_wave_dipole")
    s.objects.append(ObjectSpec("domain", cube((-pad_cells * dl, -pad_cells * dl,
                                                -reach - pad_cells * dl),
                                               (2 * pad_cells * dl, 2 * pad_cells * dl,
                                                2 * reach + 2 * pad_cells * dl)), air()))
    zc = dl + arm_cells * dl / 2
    s.thin_wires += [ThinWireSpec("arm_0", cylinder((0.0, 0.0, zc), 5e-5, arm_cells * dl, 2)),
                     ThinWireSpec("arm_1", cylinder((0.0, 0.0, -zc), 5e-5, arm_cells * dl, 2))]
    tau = dl * 30 / 6e8
    gap = cube((0.0, 0.0, -dl), (0.0, 0.0, 2 * dl))
    s.current_sources.append(VoltageSourceSpec("v_s", gap, "ZP", 50.0,
                                               Waveform("gaussian", tau, 4.5 * tau)))
    s.pmls = pml_all(pml)
    if network:
        s.line_monitors += [LineMonitorSpec("voltage", "v1", gap, "ZP"),
                            LineMonitorSpec("current", "c1", cube((0.0, 0.0, 0.0),
                                                                  (0.0, 0.0, 0.0)), "ZP")]
        s.network = NetworkSpec(list(np.arange(2e7, 2e10, 2e7)),
                                [PortSpec(1, True, 50.0, "c1", "v1")])
    if nf2ff_freqs:
        s.nf2ff = NF2FFSpec((nf2ff_distance,) * 3, list(nf2ff_freqs))
    return s


def random_boxes(n_cells: int, n_boxes: int, seed: int, edge_lo: int, edge_hi: int):
    """Box list for the dielectric-boxes scene, drawn with
    numpy.random.default_rng(seed): integer edges U[edge_lo, edge_hi] per axis,
    integer origin uniform so that the box lies inside the interior, eps_r
    U[1.5, 12], sigma_e U[0, 0.05] S/m, in generation (= painting) order."""
    rng = np.random.default_rng(seed)
    boxes = []
    for _ in range(n_boxes):
        edges = rng.integers(edge_lo, edge_hi + 1, size=3)
        edges = np.minimum(edges, n_cells)
        origin = np.array([rng.integers(0, n_cells - e + 1) for e in edges])
        eps_r = float(rng.uniform(1.5, 12.0))
        sigma = float(rng.uniform(0.0, 0.05))
        boxes.append((tuple(int(v) for v in origin), tuple(int(v) for v in edges),
                      eps_r, sigma))
    return boxes


def dielectric_boxes(n: int = 256, pml: int = 12, dl: float = 1e-3, n_boxes: int = 64,
                     steps: int = 4000, seed: int = 0, edge_lo: int = 8,
                     edge_hi: int = 40, movie_interval: int = 0) -> Scene:
    """Large vacuum/dielectric scene: n^3 cells including a `pml`-cell CPML
    (order 3, sigma_ratio 1, alpha 0..0.05, kappa_max 5), `n_boxes` random
    dielectric boxes, a z-directed one-cell CurrentSource (R = inf) at the
    centre driven by cosineModulatedGaussian(tau, 4.5 tau, 30 GHz) with
    tau = sqrt(2 ln 2)/(pi * 15 GHz), CFL 0.99."""
    interior = n - 2 * pml
    half = interior * dl / 2
    s = Scene(dl=(dl, dl, dl), cfl=0.99, steps=steps, name="dielectric_boxes")
    s.objects.append(ObjectSpec("domain", cube((-half,) * 3, (2 * half,) * 3), air()))
    for b, (o, e, eps_r, sig) in enumerate(random_boxes(interior, n_boxes, seed,
                                                        edge_lo, edge_hi)):
        org = tuple(-half + o[a] * dl for a in range(3))
        size = tuple(e[a] * dl for a in range(3))
        s.objects.append(ObjectSpec(f"box{b}", cube(org, size),
                                    Material("simple", eps_r, 1.0, sig, 0.0)))
    tau = math.sqrt(2 * math.log(2)) / (math.pi * 15e9)
    s.current_sources.append(CurrentSourceSpec(
        "dipole", cube((0.0, 0.0, 0.0), (0.0, 0.0, dl)), "ZP", math.inf,
        Waveform("cosgauss", tau, 4.5 * tau, 30e9)))
    s.pmls = pml_all(pml, order=3, sigma_ratio=1.0, alpha_min=0.0, alpha_max=0.05,
                     kappa_max=5.0)
    if movie_interval:
        s.movies.append(MovieSpec("movie_ez_xy", "EZ",
                                  cube((-half, -half, 0.0), (2 * half, 2 * half, dl)),
                                  movie_interval))
    return s


def dispersive_spheres(n: int = 384, pml: int = 10, dl: float = 5e-4, radius_cells: int = 40,
                       offsets_cells=((-100, 0), (50, 87), (50, -87)), steps: int = 6000,
                       tfsf_start: int = 20, nf2ff_distance: int = 15,
                       n_freqs: int = 32, movie_interval: int = 0,
                       media: Sequence[str] = ("drude", "lorentz", "debye")) -> Scene:
    """Dispersive ADE + TFSF + NF2FF scene: n^3 cells including a `pml`-cell
    CPML (default parameters), three spheres of radius `radius_cells` in the
    z = 0 plane (Drude eps_inf=1, wp=2pi*60 GHz, gamma=2pi*5 GHz; Lorentz
    eps_s=4, eps_inf=2, w0=2pi*40 GHz, delta=2pi*2 GHz as MLorentz(a0 =
    (eps_s-eps_inf) w0^2, a1=0, b0=w0^2, b1=2 delta, b2=1); Debye eps_s=10,
    eps_inf=3, tau=5 ps), TFSF3D(theta=45 deg, phi=30 deg, psi=0) with a
    Gaussian reaching -20 dB at 80 GHz, NF2FF at `n_freqs` frequencies in
    [10, 80] GHz, CFL 0.9.

    `media` picks which of the three spheres are present.  With all three the
    reference converts every medium to its modified-Lorentz form (one ADE
    storage for the scene), and the Debye medium's form there (b2 = 0) breaks
    the reference's own stability condition 4 b2 - b0 dt^2 >= 0: the fields
    grow without bound (about 1e50 after 1000 steps, in the reference's own
    library as in this engine).  ("drude", "lorentz") is the stable subset on
    the same storage and kernels."""
    interior = n - 2 * pml
    half = interior * dl / 2
    s = Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps, name="dispersive_spheres")
    s.objects.append(ObjectSpec("domain", cube((-half,) * 3, (2 * half,) * 3), air()))
    r = radius_cells * dl
    two_pi = 2 * math.pi
    w0 = two_pi * 40e9
    mats = [
        drude(1.0, [two_pi * 60e9], [two_pi * 5e9]),
        mlorentz(2.0, [(4.0 - 2.0) * w0 * w0], [0.0], [w0 * w0], [2 * two_pi * 2e9], [1.0]),
        debye(3.0, [10.0], [5e-12]),
    ]
    names = ("drude", "lorentz", "debye")
    for m, ((ox, oy), mat) in enumerate(zip(offsets_cells, mats)):
        if names[m] in media:
            s.objects.append(ObjectSpec(f"sphere{m}", sphere((ox * dl, oy * dl, 0.0), r), mat))
    tau = math.sqrt(math.log(10)) / (math.pi * 80e9)
    s.pmls = pml_all(pml)
    s.tfsf = TFSFSpec(tfsf_start, tfsf_start, tfsf_start, math.pi / 4, math.pi / 6, 0.0,
                      Waveform("gaussian", tau, 4.5 * tau))
    if n_freqs:
        s.nf2ff = NF2FFSpec((nf2ff_distance,) * 3,
                            list(np.linspace(10e9, 80e9, n_freqs)))
    if movie_interval:
        s.movies.append(MovieSpec("movie_ex_xy", "EX",
                                  cube((-half, -half, 0.0), (2 * half, 2 * half, dl)),
                                  movie_interval))
    return s


def adjoint_slab(nxy: int = 256, nz: int = 128, pml: int = 12, dl: float = 2e-4,
                 slab_z=(48, 64), slab_eps: float = 2.1, design=(96, 96, 16), seed: int = 2,
                 eps_range=(1.0, 12.0), freq: float = 1e12, steps: int = 5000,
                 tfsf_start: int = 16, patch: int = 16, patch_z: int = 72):
    """Adjoint inverse-design scene: nxy x nxy x nz cells including a `pml`-cell
    CPML (default parameters), dl = 0.2 mm, an eps_r = 2.1 slab over the whole
    interior in x, y at cell layers z in [slab_z), a design block of
    design[0] x design[1] x design[2] voxels (one per cell) centred in x, y
    on the same layers with eps_r U[eps_range] from numpy default_rng(seed),
    an x-polarised normal-incidence TFSF plane wave (theta = phi = psi = 0)
    carrying a cosine-modulated Gaussian at `freq` (tau = 2 / (pi freq)),
    CFL 0.99.  Returns (scene, objective) with objective = dict(field=2 (Ez),
    box_s, box_e: the patch x patch node block centred in x, y at node layer
    patch_z, freq)."""
    s = Scene(dl=(dl, dl, dl), cfl=0.99, steps=steps, name="adjoint_slab")
    n = (nxy, nxy, nz)
    half = [(n[a] - 2 * pml) * dl / 2 for a in range(3)]
    s.objects.append(ObjectSpec("domain", cube(tuple(-h for h in half),
                                               tuple(2 * h for h in half)), air()))
    # cell index c (CPML included) has its lower face at -half + (c - pml) dl
    def x0(a, c):
        return -half[a] + (c - pml) * dl
    z0, z1 = slab_z
    s.objects.append(ObjectSpec("slab", cube((-half[0], -half[1], x0(2, z0)),
                                             (2 * half[0], 2 * half[1], (z1 - z0) * dl)),
                                Material("simple", slab_eps, 1.0, 0.0, 0.0)))
    rng = np.random.default_rng(seed)
    eps = rng.uniform(eps_range[0], eps_range[1], size=design)
    c0 = [(n[a] - design[a]) // 2 for a in range(2)] + [z0 + (z1 - z0 - design[2]) // 2]
    s.objects.append(VoxelSpec("design", tuple(x0(a, c0[a]) for a in range(3)),
                               tuple(design[a] * dl for a in range(3)), eps))
    s.pmls = pml_all(pml)
    tau = 2.0 / (math.pi * freq)
    s.tfsf = TFSFSpec(tfsf_start, tfsf_start, tfsf_start, 0.0, 0.0, 0.0,
                      Waveform("cosgauss", tau, 4.5 * tau, freq))
    p0 = [(n[a] - patch) // 2 for a in range(2)]
    objective = dict(field=2, box_s=(p0[0], p0[1], patch_z),
                     box_e=(p0[0] + patch, p0[1] + patch, patch_z + 1), freq=freq)
    return s, objective


def batched_sphere_params(count: int = 96, seed: int = 1, n_lo: int = 64, n_hi: int = 224):
    """Per-scene parameters of the batched workload, drawn in this order per
    scene with numpy.random.default_rng(seed): N = round(exp(U[ln n_lo,
    ln n_hi])) cells per axis (CPML included), sphere radius U[0.1, 0.3] N
    cells, eps_r U[2, 10], TFSF theta U[0, pi], phi U[0, 2 pi), psi U[0, 2 pi)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        radius = float(rng.uniform(0.1, 0.3)) * n
        eps_r = float(rng.uniform(2.0, 10.0))
        theta = float(rng.uniform(0.0, math.pi))
        phi = float(rng.uniform(0.0, 2 * math.pi))
        psi = float(rng.uniform(0.0, 2 * math.pi))
        out.append(dict(n=n, radius_cells=radius, eps_r=eps_r, theta=theta, phi=phi, psi=psi))
    return out


def batched_sphere(n: int, radius_cells: float, eps_r: float, theta: float, phi: float,
                   psi: float, pml: int = 8, dl: float = 1e-3, tfsf_start: int = 11,
                   steps: int = 3000) -> Scene:
    """One scene of the batched workload: n^3 cells including an 8-cell CPML
    (default parameters), a centred dielectric sphere, a TFSF plane wave from
    index `tfsf_start` at (theta, phi, psi) with a Gaussian of 20 cells per
    wavelength (tau = 20 dl / 6e8, t0 = 4.5 tau, the reference examples'
    convention), CFL 0.9."""
    interior = n - 2 * pml
    half = interior * dl / 2
    s = Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps, name=f"batched_sphere_{n}")
    s.objects.append(ObjectSpec("domain", cube((-half,) * 3, (2 * half,) * 3), air()))
    s.objects.append(ObjectSpec("sphere", sphere((0.0, 0.0, 0.0), radius_cells * dl),
                                Material("simple", eps_r, 1.0, 0.0, 0.0)))
    s.pmls = pml_all(pml)
    tau = 20 * dl / 6e8
    s.tfsf = TFSFSpec(tfsf_start, tfsf_start, tfsf_start, theta, phi, psi,
                      Waveform("gaussian", tau, 4.5 * tau))
    return s


def batched_spheres(count: int = 96, seed: int = 1, steps: int = 3000, n_lo: int = 64,
                    n_hi: int = 224, **kw) -> List[Scene]:
    """The batched workload: `count` independent sphere scenes of uneven
    sizes (batched_sphere_params), each lit by its own plane wave."""
    return [batched_sphere(steps=steps, **p, **kw)
            for p in batched_sphere_params(count, seed, n_lo, n_hi)]


def microstrip_line(steps: int = 1000, n_freqs: int = 500, scale: int = 1) -> Scene:
    """The reference's microstrip-line example (test/src/examples/microstrip_line.cpp):
    cells 0.203 x 0.203 x 0.1325 mm; a 60 x 64 x 16-cell air domain on a
    6-cell eps_r = 2.2 substrate with a PEC ground plane and a 12-cell-wide
    PEC strip; a 50-ohm z-directed VoltageSource under the strip at y = 0
    driven by gaussian(tau, 4.5 tau), tau = 30 dz / 6e8; port 1 (source,
    50 ohm) from a voltage monitor under the strip and a current monitor on
    it 40 cells along; S11 at `n_freqs` frequencies in [20 MHz, 10 GHz];
    10-cell CPML on all faces but ZN (inside the domain on XN, XP, YP),
    CFL 0.9.  `scale` divides the cell counts for small parity cases."""
    dx = dy = 0.203e-3 * scale
    dz = 0.1325e-3 * scale
    q = lambda v: v // scale  # noqa: E731
    s = Scene(dl=(dx, dy, dz), cfl=0.9, steps=steps, name="microstrip_line")
    s.objects.append(ObjectSpec("domain", cube((0.0, -q(4) * dy, 0.0),
                                               (q(60) * dx, q(64) * dy, q(16) * dz)), air()))
    s.objects.append(ObjectSpec("substrate", cube((0.0, 0.0, 0.0),
                                                  (q(60) * dx, q(60) * dy, q(6) * dz)),
                                Material("simple", 2.2, 1.0, 0.0, 0.0)))
    s.pec_planes += [
        PecPlaneSpec("microstrip_0", cube((q(24) * dx, 0.0, q(6) * dz), (q(12) * dx, q(60) * dy, 0.0))),
        PecPlaneSpec("ground_0", cube((0.0, 0.0, 0.0), (q(60) * dx, q(60) * dy, 0.0))),
    ]
    tau = q(30) * dz / 6e8
    s.current_sources.append(VoltageSourceSpec(
        "v_s", cube((q(24) * dx, 0.0, 0.0), (q(12) * dx, 0.0, q(6) * dz)), "ZP", 50.0,
        Waveform("gaussian", tau, 4.5 * tau)))
    s.line_monitors += [
        LineMonitorSpec("voltage", "v1", cube((q(24) * dx, q(40) * dy, 0.0),
                                              (q(12) * dx, 0.0, q(6) * dz)), "ZP"),
        LineMonitorSpec("current", "c1", cube((q(24) * dx, q(40) * dy, q(6) * dz),
                                              (q(12) * dx, 0.0, 0.0)), "YP"),
    ]
    s.network = NetworkSpec(list(np.linspace(2e7, 10e9, n_freqs)),
                            [PortSpec(1, True, 50.0, "c1", "v1")])
    t = q(10)
    s.pmls = [PMLSpec(-t, "XN"), PMLSpec(-t, "XP"), PMLSpec(t, "YN"), PMLSpec(-t, "YP"),
              PMLSpec(t, "ZP")]
    return s
