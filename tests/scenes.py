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


ALL = {"sphere": sphere_small, "boxes": boxes_small, "dispersive": dispersive_small,
       "voxels": voxels_small}
