"""Small variants of the three benchmark scenes: the same geometry rules at
sizes the oracle runs in seconds."""
from xfdtd_core_b200 import scene as S


def sphere_small(steps=120, **kw):
    base = dict(steps=steps, dl=0.35 / 20, radius=0.07, pml=6, tfsf_start=9, movie_interval=10)
    base.update(kw)
    return S.dielectric_sphere(**base)


def boxes_small(steps=120, **kw):
    base = dict(n=40, pml=8, n_boxes=8, edge_lo=3, edge_hi=10, steps=steps, movie_interval=0)
    base.update(kw)
    return S.dielectric_boxes(**base)


def dispersive_small(steps=120, **kw):
    base = dict(n=48, pml=6, radius_cells=5, offsets_cells=((-10, 0), (5, 9), (5, -9)),
                steps=steps, tfsf_start=9, nf2ff_distance=8, n_freqs=4, movie_interval=0)
    base.update(kw)
    return S.dispersive_spheres(**base)


def dispersive_stable_small(steps=120, **kw):
    """The dispersive scene with its Drude and Lorentz spheres only: the same
    modified-Lorentz ADE storage and kernels, without the Debye sphere whose
    modified-Lorentz form is unstable in the reference's scheme."""
    kw.setdefault("media", ("drude", "lorentz"))
    return dispersive_small(steps=steps, **kw)


def voxels_small(steps=120, **kw):
    """The adjoint scene's geometry at 40 x 40 x 32: slab, 8 x 8 x 3 design
    voxels, normal-incidence TFSF, Ez patch objective."""
    base = dict(nxy=40, nz=32, pml=6, dl=2e-4, slab_z=(12, 18), design=(8, 8, 3),
                tfsf_start=8, patch=4, patch_z=22, steps=steps, freq=3e11)
    base.update(kw)
    return S.adjoint_slab(**base)[0]


def voxels_objective(**kw):
    base = dict(nxy=40, nz=32, pml=6, dl=2e-4, slab_z=(12, 18), design=(8, 8, 3),
                tfsf_start=8, patch=4, patch_z=22, freq=3e11)
    base.update(kw)
    return S.adjoint_slab(**base)[1]


def lumped_small(steps=120, n=32, pml=6, dl=1e-3):
    """Every lumped element in a CPML-bounded air box: a 50-ohm z-directed
    voltage source (two cells) at the centre with a 100-ohm resistor sharing
    its upper node (the later element's coefficients win there), a resistor,
    an x-directed capacitor, a z-directed inductor, a y-directed current
    source with R = 200 ohm, and voltage / current monitors on them."""
    import math
    interior = n - 2 * pml
    half = interior * dl / 2
    sc = S.Scene(dl=(dl, dl, dl), cfl=0.99, steps=steps, name="lumped")
    sc.objects.append(S.ObjectSpec("domain", S.cube((-half,) * 3, (2 * half,) * 3), S.air()))
    tau = math.sqrt(2 * math.log(2)) / (math.pi * 15e9)
    wave = S.Waveform("cosgauss", tau, 4.5 * tau, 30e9)
    sc.current_sources += [
        S.VoltageSourceSpec("vs", S.cube((0.0, 0.0, -dl), (0.0, 0.0, 2 * dl)), "ZP", 50.0, wave),
        S.CurrentSourceSpec("is", S.cube((-3 * dl, -2 * dl, 2 * dl), (0.0, 2 * dl, 0.0)), "YN",
                            200.0, wave),
    ]
    sc.lumped_elements += [
        S.LumpedSpec("resistor", "r_top", S.cube((0.0, 0.0, 0.0), (0.0, 0.0, dl)), "Z", 100.0),
        S.LumpedSpec("resistor", "r1", S.cube((4 * dl, 0.0, -dl), (0.0, 0.0, 2 * dl)), "Z", 100.0),
        S.LumpedSpec("capacitor", "c1", S.cube((-5 * dl, 2 * dl, 0.0), (2 * dl, 0.0, 0.0)), "X",
                     1e-12),
        S.LumpedSpec("inductor", "l1", S.cube((0.0, -4 * dl, -dl), (dl, 0.0, 2 * dl)), "Z", 2e-9),
    ]
    sc.pmls = S.pml_all(pml)
    sc.line_monitors = [
        S.LineMonitorSpec("voltage", "v_vs", S.cube((0.0, 0.0, -dl), (0.0, 0.0, 2 * dl)), "ZP"),
        S.LineMonitorSpec("voltage", "v_l1", S.cube((0.0, -4 * dl, -dl), (dl, 0.0, 2 * dl)), "ZP"),
        S.LineMonitorSpec("current", "i_vs", S.cube((-dl, -dl, -dl), (2 * dl, 2 * dl, 2 * dl)),
                          "ZP"),
        S.LineMonitorSpec("current", "i_r1",
                          S.cube((3 * dl, -dl, -dl), (2 * dl, 2 * dl, 2 * dl)), "ZP"),
    ]
    return sc


def microstrip_small(steps=150, **kw):
    """The microstrip-line example (PEC planes, voltage source, port, network)
    at half the cell count."""
    base = dict(steps=steps, n_freqs=40, scale=2)
    base.update(kw)
    return S.microstrip_line(**base)


ALL = {"sphere": sphere_small, "boxes": boxes_small, "dispersive": dispersive_small,
       "dispersive_stable": dispersive_stable_small, "voxels": voxels_small,
       "lumped": lumped_small, "microstrip": microstrip_small}


def wires_small(steps=120, n=30, pml=6, dl=1e-3):
    """Thin wires along all three axes in a CPML-bounded air box: a z dipole
    fed by a 50-ohm voltage source in its gap, an x wire and a y wire off to
    the sides (each with the radius below half a cell), a Gaussian voltage,
    and an NF2FF surface at two frequencies."""
    import math
    interior = n - 2 * pml
    half = interior * dl / 2
    sc = S.Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps, name="wires")
    sc.objects.append(S.ObjectSpec("domain", S.cube((-half,) * 3, (2 * half,) * 3), S.air()))
    sc.thin_wires += [
        S.ThinWireSpec("z_up", S.cylinder((0.0, 0.0, 3.5 * dl), 1e-4, 5 * dl, 2)),
        S.ThinWireSpec("z_dn", S.cylinder((0.0, 0.0, -3.5 * dl), 1e-4, 5 * dl, 2)),
        S.ThinWireSpec("x_w", S.cylinder((0.0, 5 * dl, -2 * dl), 2e-4, 6 * dl, 0)),
        S.ThinWireSpec("y_w", S.cylinder((-5 * dl, 0.0, 2 * dl), 5e-5, 6 * dl, 1)),
    ]
    tau = 20 * dl / 6e8
    sc.current_sources.append(S.VoltageSourceSpec(
        "v_s", S.cube((0.0, 0.0, -dl), (0.0, 0.0, 2 * dl)), "ZP", 50.0,
        S.Waveform("gaussian", tau, 4.5 * tau)))
    sc.pmls = S.pml_all(pml)
    sc.nf2ff = S.NF2FFSpec((3, 3, 3), [2e10, 5e10])
    return sc
