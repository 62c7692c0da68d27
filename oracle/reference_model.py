"""ORACLE -- TEST INFRASTRUCTURE ONLY.  PARITY UNPINNED.

numpy restatement of EMinsight/XFDTD_CORE's initialisation (grid generation,
object painting, edge/face averaging, the 18 Yee coefficients, CPML grading,
TFSF incident grid, lumped elements, PEC planes, ADE coefficients, NF2FF
phasors, movie, voltage and current monitors, network S-parameters) driving
the C per-step routines in ``xfd_oracle.c``.  The CUDA engine's parity tests
compare against it, and it is the timed CPU baseline; the product never
imports it.

The reference publishes no golden vectors and cannot be compiled here (its
only dependency, xtensor <= 0.25.0 with xtl, is absent and there is no
network), so this restatement is not pinned to outputs of the reference
itself.  Each step cites the reference lines it restates; the xtensor view
expressions map one to one onto numpy slicing, including the
evaluate-right-hand-side-first semantics of an assignment to an overlapping
view (src/calculation_param/calculation_param.cpp:55-63).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libxfd_oracle.so")

# include/xfdtd/common/constant.h:11-18
PI = math.pi
EPSILON_0 = 8.854187817e-12
MU_0 = 4 * PI * 1e-7
C_0 = 1 / math.sqrt(EPSILON_0 * MU_0)
SIGMA_E_ZERO = 1e-20  # constant.h:17, material.h:40
SIGMA_M_ZERO = 1e-20

AXIS = {"X": 0, "Y": 1, "Z": 2}
DIR = {"XN": (0, True), "XP": (0, False), "YN": (1, True), "YP": (1, False),
       "ZN": (2, True), "ZP": (2, False)}


def tan_a(c: int) -> int:
    return (c + 1) % 3


def tan_b(c: int) -> int:
    return (c + 2) % 3


def build_library(force: bool = False) -> str:
    """Compiles xfd_oracle.c (gcc, OpenMP, no FMA contraction) into _build/."""
    src = os.path.join(HERE, "xfd_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(BUILD, exist_ok=True)
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                           "-fPIC", "-shared", "-o", LIB_PATH, src])
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        build_library()
        _LIB = ctypes.CDLL(LIB_PATH)
        _LIB.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int64]
        _LIB.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64]
        _LIB.orc_set_num_threads.argtypes = [ctypes.c_int]
        _LIB.orc_num_threads.restype = ctypes.c_int
    return _LIB


# ---------------------------------------------------------------------------
# ctypes mirrors of the C structs
# ---------------------------------------------------------------------------
_dp = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64


class _Arr(ctypes.Structure):
    _fields_ = [("p", _dp), ("n", _i64 * 3)]


class _Yee(ctypes.Structure):
    _fields_ = [("nx", _i64), ("ny", _i64), ("nz", _i64),
                ("e", _Arr * 3), ("h", _Arr * 3), ("ce", _Arr * 3), ("ceh_a", _Arr * 3),
                ("ceh_b", _Arr * 3), ("ch", _Arr * 3), ("che_a", _Arr * 3),
                ("che_b", _Arr * 3)]


class _Ade(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("np", _i64),
                ("cjj", _dp), ("cjjp", _dp), ("cjen", _dp), ("cje", _dp), ("cjep", _dp),
                ("cjsumj", _dp), ("cjsumjp", _dp), ("cejsum", _dp), ("ceep", _dp),
                ("eprev", _dp * 3), ("j", _dp * 3), ("jprev", _dp * 3)]


class _Pml(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", _i64), ("e_start", _i64), ("h_start", _i64),
                ("task_s", _i64 * 3), ("task_e", _i64 * 3),
                ("a_e", _dp), ("b_e", _dp), ("a_h", _dp), ("b_h", _dp),
                ("c_psi", _Arr * 4), ("psi", _Arr * 4)]


class _Tfsf(ctypes.Structure):
    _fields_ = [("is_", _i64), ("ie", _i64), ("js", _i64), ("je", _i64), ("ks", _i64),
                ("ke", _i64), ("nt", _i64), ("aux", _i64), ("e_inc", _dp), ("h_inc", _dp),
                ("p_int", _dp * 3), ("p_half", _dp * 3), ("ca", ctypes.c_double * 3),
                ("cb", ctypes.c_double * 3), ("te", ctypes.c_double * 3),
                ("th", ctypes.c_double * 3), ("xo", _i64), ("nxl", _i64)]


class _Lumped(ctypes.Structure):
    _fields_ = [("comp", ctypes.c_int), ("s", _i64 * 3), ("e", _i64 * 3), ("coff", _dp),
                ("wave", _dp), ("cecjc", _dp), ("j", _dp)]


class _Nf2ff(ctypes.Structure):
    _fields_ = [("nf", _i64), ("nt", _i64), ("task_s", (_i64 * 3) * 6),
                ("task_e", (_i64 * 3) * 6), ("te", _dp), ("th", _dp), ("acc", _dp),
                ("off", ctypes.POINTER(_i64))]


class _Nf2ffTd(ctypes.Structure):
    _fields_ = [("task_s", (_i64 * 3) * 6), ("task_e", (_i64 * 3) * 6), ("delay", _dp),
                ("ds", _dp), ("prev", _dp), ("pot", _dp), ("P", _i64), ("n_bins", _i64)]


class _Sim(ctypes.Structure):
    _fields_ = [("yee", ctypes.POINTER(_Yee)), ("ade", ctypes.POINTER(_Ade)),
                ("pml", ctypes.POINTER(_Pml)), ("n_pml", _i64),
                ("tfsf", ctypes.POINTER(_Tfsf)), ("lumped", ctypes.POINTER(_Lumped)),
                ("n_lumped", _i64), ("nf2ff", ctypes.POINTER(_Nf2ff)),
                ("nf2ff_td", ctypes.POINTER(_Nf2ffTd))]


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def _arr(a: np.ndarray) -> _Arr:
    s = _Arr()
    s.p = _ptr(a)
    for d in range(3):
        s.n[d] = a.shape[d]
    return s


# ---------------------------------------------------------------------------
# Geometry helpers
# ---------------------------------------------------------------------------

def xround(x: float) -> int:
    """std::round (half away from zero) for the non-negative grid counts."""
    return int(math.floor(x + 0.5))


def linspace(start: float, stop: float, n: int) -> np.ndarray:
    """xt::linspace(start, stop, n) with endpoint: start + i*step, last = stop."""
    return np.linspace(start, stop, n)


class _Cube:
    def __init__(self, origin, size):
        self.origin = np.array(origin, dtype=np.float64)
        self.size = np.array(size, dtype=np.float64)
        self.end = self.origin + self.size  # Cube::updateEnd (src/shape/cube.cpp)


def wrapped_cube(shape) -> _Cube:
    if shape.kind == "cube":
        return _Cube(shape.origin, shape.size)
    if shape.kind == "cylinder":
        # Cylinder::wrappedCube (src/shape/cylinder.cpp:72-98)
        c = np.array(shape.origin, dtype=np.float64)
        half = np.array([shape.radius] * 3)
        half[shape.axis] = shape.height / 2
        return _Cube(c - half, 2 * half)
    c = np.array(shape.origin, dtype=np.float64)
    r = shape.radius
    # Sphere::wrappedCube (src/shape/sphere.cpp:34-37)
    return _Cube(c - np.array([r, r, r]), np.array([r * 2, r * 2, r * 2]))


def float_le(lhs, rhs, eps):
    """floatCompare(lhs, rhs, LessEqual, eps) (src/include/util/float_compare.h:20-42)."""
    return (np.abs(lhs - rhs) <= eps) | (lhs < rhs)


def inside(shape, x, y, z, eps):
    """Shape::isInside (src/shape/sphere.cpp:29-32, src/shape/cube.cpp:58-73)."""
    if shape.kind == "sphere":
        c = shape.origin
        dx, dy, dz = x - c[0], y - c[1], z - c[2]
        d = np.sqrt(dx * dx + dy * dy + dz * dz)
        return float_le(d, shape.radius, eps)
    if shape.kind == "cylinder":
        # Cylinder::isInside (src/shape/cylinder.cpp:44-66): inside the wrapped
        # cube, then within the radius of the axis (floatCompare's 1e-8)
        cb = wrapped_cube(shape)
        box = (float_le(cb.origin[0], x, eps) & float_le(x, cb.end[0], eps) &
               float_le(cb.origin[1], y, eps) & float_le(y, cb.end[1], eps) &
               float_le(cb.origin[2], z, eps) & float_le(z, cb.end[2], eps))
        c = shape.origin
        d = [x - c[0], y - c[1], z - c[2]]
        u, v = [(1, 2), (0, 2), (0, 1)][shape.axis]
        dis = np.sqrt(d[u] ** 2 + d[v] ** 2)
        return box & float_le(dis, shape.radius, 1e-8)
    cb = _Cube(shape.origin, shape.size)
    return (float_le(cb.origin[0], x, eps) & float_le(x, cb.end[0], eps) &
            float_le(cb.origin[1], y, eps) & float_le(y, cb.end[1], eps) &
            float_le(cb.origin[2], z, eps) & float_le(z, cb.end[2], eps))


class RefSimulation:
    """One ``xfdtd::Simulation`` with the reference's init and step order."""

    def __init__(self, scene, threads: int = 0):
        self.scene = scene
        self.threads = threads
        self.movie_frames: Dict[str, List[np.ndarray]] = {}
        self._keep = []  # keeps ctypes-referenced arrays alive
        self._init()

    @classmethod
    def from_arrays(cls, n, e, h, ce, ceh_a, ceh_b, ch, che_a, che_b, pml=(), tfsf=None,
                    lumped=(), ade=None, nf2ff=None, threads: int = 0):
        """Oracle over explicit fields and the 18 coefficient arrays (reference
        shapes), for kernel-level checks that bypass the scene init.  `pml`
        entries are dicts with the keys produced by _pml()."""
        self = cls.__new__(cls)
        self.scene = None
        self.threads = threads
        self.movie_frames = {}
        self.movies = []
        self.field_times = []
        self._keep = []
        self.nx, self.ny, self.nz = n
        f = lambda arrs: [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        self.e, self.h = f(e), f(h)
        self.ce, self.ceh_a, self.ceh_b = f(ce), f(ceh_a), f(ceh_b)
        self.ch, self.che_a, self.che_b = f(ch), f(che_a), f(che_b)
        self.pml = list(pml)
        self.tfsf = tfsf
        self.lumped = list(lumped)
        self.ade = ade
        self.nf2ff = nf2ff
        self.nf2ff_td = None
        self.line_monitors = []
        self._bind()
        self.t = 0
        return self

    # ------------------------------------------------------------------ grid
    def _grid(self):
        sc = self.scene
        dx, dy, dz = sc.dl
        shapes = [o.shape for o in sc.objects] + \
            [w.shape for w in getattr(sc, "thin_wires", [])] + \
            [c.shape for c in sc.current_sources] + \
            [c.shape for c in getattr(sc, "lumped_elements", [])] + \
            [c.shape for c in getattr(sc, "pec_planes", [])]
        lo = np.full(3, np.finfo(np.float64).max)
        hi = np.full(3, np.finfo(np.float64).min)
        for s in shapes:  # Shape::makeWrappedCube (src/shape/shape.cpp:8-38)
            cb = wrapped_cube(s)
            lo = np.minimum(lo, cb.origin)
            hi = np.maximum(hi, cb.end)
        dom = _Cube(lo, hi - lo)
        mn, mx = dom.origin.copy(), dom.end.copy()
        based = (dx, dy, dz)
        for p in sc.pmls:  # extendDomain (src/grid_space/grid_space_generator.cpp:36-99)
            a, neg = DIR[p.direction]
            if p.thickness < 0:
                continue
            if neg:
                mn[a] -= p.thickness * based[a]
            else:
                mx[a] += p.thickness * based[a]
        dom = _Cube(mn, mx - mn)
        # generateGridSpace3D (grid_space_generator.cpp:183-217)
        n = []
        nodes = []
        for a in range(3):
            lo_a, hi_a = dom.origin[a], dom.end[a]
            na = xround((hi_a - lo_a) / based[a])
            if na <= 1:
                raise ValueError("GridSpace is too small")
            hi_a = lo_a + based[a] * na
            region_end = lo_a + (hi_a - lo_a)
            nodes.append(linspace(lo_a, region_end, na + 1))
            n.append(na)
        self.nx, self.ny, self.nz = n
        self.e_node = nodes
        # correctGridSpaceForOne (src/grid_space/grid_space.cpp:517-544)
        self.h_node = [(e[:-1] + e[1:]) / 2 for e in nodes]
        self.e_size = [e[1:] - e[:-1] for e in nodes]
        self.h_size = []
        for a in range(3):
            e = nodes[a]
            tmp = np.concatenate([[e[0] - based[a] / 2], self.h_node[a], [e[-1] + based[a] / 2]])
            self.h_size.append(tmp[1:] - tmp[:-1])
        self.min_d = [float(np.min(s)) for s in self.e_size]
        self.based = based
        # TimeParam::calculateDt (src/calculation_param/time_param.cpp:10-13)
        ddx, ddy, ddz = self.min_d
        self.dt = sc.cfl / (C_0 * math.sqrt(1.0 / (ddx * ddx) + 1.0 / (ddy * ddy) +
                                            1.0 / (ddz * ddz)))
        # GridSpace::eps (grid_space.cpp:459-468)
        self.eps = min(self.min_d) / 1000

    def nearest(self, a: int, x: float) -> int:
        """handleTransform*WithoutCheck: argmin |e_node - x| (grid_space.cpp:505-515)."""
        return int(np.argmin(np.abs(self.e_node[a] - x)))

    def grid_box(self, shape):
        """GridSpace::getGridBoxWithoutCheck on the shape's wrapped cube."""
        cb = wrapped_cube(shape)
        o = [self.nearest(a, cb.origin[a]) for a in range(3)]
        e = [self.nearest(a, cb.end[a]) for a in range(3)]
        return o, e

    # -------------------------------------------------------------- materials
    def _materials(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        shp_e = [(nx, ny + 1, nz + 1), (nx + 1, ny, nz + 1), (nx + 1, ny + 1, nz)]
        shp_h = [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]
        self.shp_e, self.shp_h = shp_e, shp_h
        # MaterialParam::allocate (src/calculation_param/material_param.cpp:365-393)
        eps = [np.full(s, EPSILON_0) for s in shp_e]
        sig_e = [np.full(s, SIGMA_E_ZERO) for s in shp_e]
        mu = [np.full(s, MU_0) for s in shp_h]
        sig_m = [np.full(s, SIGMA_M_ZERO) for s in shp_h]
        self.cell_material = np.zeros((nx, ny, nz), dtype=np.int32)
        mats = []
        painters = [(o.shape, o.material) for o in self.scene.objects]
        voxels = [o if hasattr(o, "voxel_index") else None for o in self.scene.objects]
        from_air = __import__("xfdtd_core_b200.scene", fromlist=["air"]).air
        wires = list(getattr(self.scene, "thin_wires", []))
        painters += [(w.shape, from_air()) for w in wires]
        voxels += [None] * len(wires)
        lumped = list(self.scene.current_sources) + list(getattr(self.scene, "lumped_elements", []))
        painters += [(c.shape, from_air()) for c in lumped]
        voxels += [None] * len(lumped)
        # Simulation::correctMaterialSpace (src/simulation/simulation.cpp:608-636)
        # -> Object::defaultCorrectMaterialSpace (src/object/object.cpp:114-198)
        for index, (shape, mat) in enumerate(painters):
            if mat.kind == "simple":
                er, mr, se, sm = mat.eps_r, mat.mu_r, mat.sigma_e, mat.sigma_m
            else:  # dispersive factories carry ElectroMagneticProperty::air()
                er, mr, se, sm = 1.0, 1.0, SIGMA_E_ZERO, SIGMA_M_ZERO
            # ElectroMagneticProperty ctor (src/material/material.cpp:11-26)
            e_val, m_val = er * EPSILON_0, mr * MU_0
            se = SIGMA_E_ZERO if se == 0 else se
            sm = SIGMA_M_ZERO if sm == 0 else sm
            # Only cells whose centre lies within the shape's wrapped cube
            # (+ tolerance) can test inside; the reference evaluates the same
            # predicate on every cell.
            cb = wrapped_cube(shape)
            lo = [int(np.searchsorted(self.h_node[a], cb.origin[a] - 2 * self.eps, "left"))
                  for a in range(3)]
            hi = [int(np.searchsorted(self.h_node[a], cb.end[a] + 2 * self.eps, "right"))
                  for a in range(3)]
            if any(hi[a] <= lo[a] for a in range(3)):
                mats.append(mat)
                continue
            X, Y, Z = np.meshgrid(self.h_node[0][lo[0]:hi[0]], self.h_node[1][lo[1]:hi[1]],
                                  self.h_node[2][lo[2]:hi[2]], indexing="ij")
            sub = inside(shape, X, Y, Z, self.eps)
            mask = np.zeros((nx, ny, nz), dtype=bool)
            mask[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = sub
            if voxels[index] is not None:
                # A per-voxel permittivity block (an Object overriding
                # correctMaterialSpace, include/xfdtd/object/object.h:47):
                # each painted cell takes the eps_r of the voxel holding its
                # centre.
                v = voxels[index]
                qi = [v.voxel_index(a, self.h_node[a][lo[a]:hi[a]]) for a in range(3)]
                QI, QJ, QK = np.meshgrid(*qi, indexing="ij")
                e_val = np.zeros((nx, ny, nz))
                e_val[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = (
                    np.asarray(v.eps_r, dtype=np.float64)[QI, QJ, QK] * EPSILON_0)
                e_val = e_val[mask]
            for c in range(3):
                eps[c][:nx, :ny, :nz][mask] = e_val
                sig_e[c][:nx, :ny, :nz][mask] = se
                mu[c][:nx, :ny, :nz][mask] = m_val
                sig_m[c][:nx, :ny, :nz][mask] = sm
            self.cell_material[mask] = index
            mats.append(mat)
        self.materials = mats
        # CalculationParam::generateMaterialSpaceParam (calculation_param.cpp:43-168)
        ex, ey, ez = eps
        ex[0:nx, 1:ny, 1:nz] = 0.25 * (ex[0:nx, 1:ny, 1:nz] + ex[0:nx, 0:ny - 1, 1:nz] +
                                       ex[0:nx, 1:ny, 0:nz - 1] + ex[0:nx, 0:ny - 1, 0:nz - 1])
        ey[1:nx, 0:ny, 1:nz] = 0.25 * (ey[1:nx, 0:ny, 1:nz] + ey[0:nx - 1, 0:ny, 1:nz] +
                                       ey[1:nx, 0:ny, 0:nz - 1] + ey[0:nx - 1, 0:ny, 0:nz - 1])
        ez[1:nx, 1:ny, 0:nz] = 0.25 * (ez[1:nx, 1:ny, 0:nz] + ez[0:nx - 1, 1:ny, 0:nz] +
                                       ez[1:nx, 0:ny - 1, 0:nz] + ez[0:nx - 1, 0:ny - 1, 0:nz])
        mx, my, mz = mu
        mx[1:nx, :, :] = 2 * mx[1:nx, 0:ny, 0:nz] * mx[0:nx - 1, 0:ny, 0:nz] / (
            mx[1:nx, 0:ny, 0:nz] + mx[0:nx - 1, 0:ny, 0:nz])
        my[:, 1:ny, :] = 2 * my[0:nx, 1:ny, 0:nz] * my[0:nx, 0:ny - 1, 0:nz] / (
            my[0:nx, 1:ny, 0:nz] + my[0:nx, 0:ny - 1, 0:nz])
        mz[:, :, 1:nz] = 2 * mz[0:nx, 0:ny, 1:nz] * mz[0:nx, 0:ny, 0:nz - 1] / (
            mz[0:nx, 0:ny, 1:nz] + mz[0:nx, 0:ny, 0:nz - 1])
        sx, sy, sz = sig_e
        sx[0:nx, 1:ny, 1:nz] = 0.25 * (sx[0:nx, 1:ny, 1:nz] + sx[0:nx, 0:ny - 1, 1:nz] +
                                       sx[0:nx, 1:ny, 0:nz - 1] + sx[0:nx, 0:ny - 1, 0:nz - 1])
        sy[1:nx, 0:ny, 1:nz] = 0.25 * (sy[1:nx, 0:ny, 1:nz] + sy[0:nx - 1, 0:ny, 1:nz] +
                                       sy[1:nx, 0:ny, 0:nz - 1] + sy[0:nx - 1, 0:ny, 0:nz - 1])
        sz[1:nx, 1:ny, 0:nz] = 0.25 * (sz[1:nx, 1:ny, 0:nz] + sz[0:nx - 1, 1:ny, 0:nz] +
                                       sz[1:nx, 0:ny - 1, 0:nz] + sz[0:nx - 1, 0:ny - 1, 0:nz])
        qx, qy, qz = sig_m
        qx[1:nx, :, :] = 2 * qx[1:nx, 0:ny, 0:nz] * qx[0:nx - 1, 0:ny, 0:nz] / (
            qx[1:nx, 0:ny, 0:nz] + qx[0:nx - 1, 0:ny, 0:nz])
        qy[:, 1:ny, :] = 2 * qy[0:nx, 1:ny, 0:nz] * qy[0:nx, 0:ny - 1, 0:nz] / (
            qy[0:nx, 1:ny, 0:nz] + qy[0:nx, 0:ny - 1, 0:nz])
        qz[:, :, 1:nz] = 2 * qz[0:nx, 0:ny, 1:nz] * qz[0:nx, 0:ny, 0:nz - 1] / (
            qz[0:nx, 0:ny, 1:nz] + qz[0:nx, 0:ny, 0:nz - 1])
        # PecPlane::correctMaterialSpace (src/object/lumped_element/pec_plane.cpp:12-66)
        # after the averaging (src/simulation/simulation.cpp:628-635): the PEC
        # sigma_e (ElectroMagneticProperty::pec, src/material/material.cpp:32-34)
        # on the plane's two tangential E components.
        for pp in getattr(self.scene, "pec_planes", []):
            (i0, j0, k0), (i1, j1, k1) = self.grid_box(pp.shape)
            if i0 == i1:
                sig_e[1][i0, j0:j1, k0:k1 + 1] = 1e10
                sig_e[2][i0, j0:j1 + 1, k0:k1] = 1e10
            elif j0 == j1:
                sig_e[2][i0:i1 + 1, j0, k0:k1] = 1e10
                sig_e[0][i0:i1, j0, k0:k1 + 1] = 1e10
            elif k0 == k1:
                sig_e[0][i0:i1, j0:j1 + 1, k0] = 1e10
                sig_e[1][i0:i1 + 1, j0:j1, k0] = 1e10
            else:
                raise ValueError(f"{pp.name} PecPlane is not a plane!")
        self.eps_arr, self.sig_e_arr, self.mu_arr, self.sig_m_arr = eps, sig_e, mu, sig_m

    # ----------------------------------------------------------- coefficients
    def _coefficients(self):
        """CalculationParam::calculateCoefficient (calculation_param.cpp:170-264)."""
        dt = self.dt
        hs, es = self.h_size, self.e_size
        ce, ceh_a, ceh_b, ch, che_a, che_b = [], [], [], [], [], []
        for c in range(3):
            A, B = tan_a(c), tan_b(c)
            # E_c lives on e-size along c and h-size across; da = d along A, db = d along B.
            sizes = [hs[0], hs[1], hs[2]]
            sizes[c] = es[c]
            grids = np.meshgrid(*sizes, indexing="ij")
            da, db = grids[A], grids[B]
            eps, sig = self.eps_arr[c], self.sig_e_arr[c]
            cece = (2 * eps - dt * sig) / (2 * eps + dt * sig)
            cecha = -(2 * dt / db) / (2 * eps + sig * dt)
            cechb = (2 * dt / da) / (2 * eps + sig * dt)
            ce.append(np.ascontiguousarray(cece))
            ceh_a.append(np.ascontiguousarray(cecha))
            ceh_b.append(np.ascontiguousarray(cechb))
            sizes = [es[0], es[1], es[2]]
            sizes[c] = hs[c]
            grids = np.meshgrid(*sizes, indexing="ij")
            da, db = grids[A], grids[B]
            mu, sm = self.mu_arr[c], self.sig_m_arr[c]
            chch = (2 * mu - dt * sm) / (2 * mu + dt * sm)
            chcea = (2 * dt / db) / (2 * mu + sm * dt)
            chceb = -(2 * dt / da) / (2 * mu + sm * dt)
            ch.append(np.ascontiguousarray(chch))
            che_a.append(np.ascontiguousarray(chcea))
            che_b.append(np.ascontiguousarray(chceb))
        self.ce, self.ceh_a, self.ceh_b = ce, ceh_a, ceh_b
        self.ch, self.che_a, self.che_b = ch, che_a, che_b

    # ------------------------------------------------------------ thin wires
    def _thin_wires(self):
        """ThinWire::init / correctUpdateCoefficient (src/object/thin_wire.cpp:12-152):
        on the wire's nodes the E along the wire gets ce = ceh_a = ceh_b = 0;
        the H coefficients the reference scales next to the wire take
        k 2 / ln(d / r): chyex, chzex for an x wire; chzey, chxey for y;
        chxey, chyex for z."""
        dx, dy, dz = self.based
        for w in getattr(self.scene, "thin_wires", []):
            sh = w.shape
            ax, r = sh.axis, sh.radius
            u, v = (ax + 1) % 3, (ax + 2) % 3
            if not (r < self.based[u] / 2 and r < self.based[v] / 2):
                raise ValueError("ThinWire::init: wire is not thin enough")
            (i_s, j_s, k_s), (i_e, j_e, k_e) = self.grid_box(sh)
            if ax == 0:
                sl = (slice(i_s, i_e), j_s, k_s)
            elif ax == 1:
                sl = (i_s, slice(j_s, j_e), k_s)
            else:
                sl = (i_s, j_s, slice(k_s, k_e))
            for arr in (self.ce, self.ceh_a, self.ceh_b):
                arr[ax][sl] = 0
            # che_a / che_b of component c multiply E_{c+1} / E_{c+2}:
            # chxey = che_a[0], chyex = che_b[1], chzex = che_a[2], chzey = che_b[2]
            if ax == 0:
                khy = dz * math.atan(dy / dy) / dy
                khz = dy * math.atan(dz / dy) / dz
                v1 = self.che_b[1][i_s:i_e, j_s, k_s - 1:k_s + 1]
                self.che_b[1][i_s:i_e, j_s, k_s - 1:k_s + 1] = khy * 2 * v1 / math.log(dz / r)
                v2 = self.che_a[2][i_s:i_e, j_s - 1:j_s + 1, k_s]
                self.che_a[2][i_s:i_e, j_s - 1:j_s + 1, k_s] = khz * 2 * v2 / math.log(dy / r)
            elif ax == 1:
                khz = dx * math.atan(dz / dx) / dz
                khx = dz * math.atan(dx / dz) / dx
                v1 = self.che_b[2][i_s - 1:i_s + 1, j_s:j_e, k_s]
                self.che_b[2][i_s - 1:i_s + 1, j_s:j_e, k_s] = khz * 2 * v1 / math.log(dx / r)
                v2 = self.che_a[0][i_s, j_s:j_e, k_s - 1:k_s + 1]
                self.che_a[0][i_s, j_s:j_e, k_s - 1:k_s + 1] = khx * 2 * v2 / math.log(dz / r)
            else:
                khx = dy * math.atan(dx / dy) / dx
                khy = dx * math.atan(dy / dx) / dy
                v1 = self.che_a[0][i_s, j_s - 1:j_s + 1, k_s:k_e]
                self.che_a[0][i_s, j_s - 1:j_s + 1, k_s:k_e] = khx * 2 * v1 / math.log(dy / r)
                v2 = self.che_b[1][i_s - 1:i_s + 1, j_s, k_s:k_e]
                self.che_b[1][i_s - 1:i_s + 1, j_s, k_s:k_e] = khy * 2 * v2 / math.log(dx / r)

    # ------------------------------------------------------- current sources
    def _current_sources(self):
        """Lumped elements in object order (current and voltage sources, then
        resistors, capacitors, inductors): ::init and ::correctUpdateCoefficient
        of src/object/lumped_element/current_source.cpp:40-165,
        voltage_source.cpp:47-163, resistor.cpp:27-127, capacitor.cpp:16-112,
        inductor.cpp:23-105, computed from the eps / sigma arrays."""
        self.lumped = []
        dt = self.dt
        elements = list(self.scene.current_sources) + \
            list(getattr(self.scene, "lumped_elements", []))
        for el in elements:
            kind = getattr(el, "kind", "current")
            if kind in ("current", "voltage"):
                axis, neg = DIR[el.direction]
            else:
                axis, neg = "XYZ".index(el.axis), False
            o, e = self.grid_box(el.shape)
            # LumpedElement::rangeX/Y/Z (include/xfdtd/object/lumped_element/lumped_element.h:79-104)
            s = list(o)
            en = [e[a] if a == axis else e[a] + 1 for a in range(3)]
            size = [e[a] - o[a] for a in range(3)]
            A, B = tan_a(axis), tan_b(axis)
            na, nb, nc = size[A] + 1, size[B] + 1, size[axis]
            sizes = [self.h_size[0], self.h_size[1], self.h_size[2]]
            sizes[axis] = self.e_size[axis]
            sl = [slice(s[a], en[a]) for a in range(3)]
            g = np.meshgrid(sizes[0][sl[0]], sizes[1][sl[1]], sizes[2][sl[2]], indexing="ij")
            d_a, d_b, d_c = g[A], g[B], g[axis]
            eps = self.eps_arr[axis][sl[0], sl[1], sl[2]]
            sig = self.sig_e_arr[axis][sl[0], sl[1], sl[2]]
            if kind == "inductor":
                ind = el.value if el.value != 0 else 1e-10
                ind_factor = ind * na * nb / nc
                self.lumped.append({
                    "comp": axis, "s": s, "e": en,
                    "coff": np.ascontiguousarray(dt * d_c / (ind_factor * d_a * d_b)),
                    "cecjc": np.ascontiguousarray(-(2 * dt) / (2 * eps + dt * sig)),
                    "j": np.zeros(d_c.shape)})
                continue
            sign = 1.0
            if kind == "capacitor":
                cap_factor = el.value * nc / (nc * nb)
                beta = 2 * cap_factor * d_c / (d_a * d_b)
                sign = -1.0
            else:
                r = el.resistance if kind in ("current", "voltage") else el.value
                if r == 0:
                    r = 1e-10 if kind == "resistor" else 1e-20
                res_factor = r * na * nb / nc
                if kind == "voltage":
                    alpha = d_a * d_b * res_factor
                    beta = dt * d_c / alpha
                else:
                    beta = (dt * d_c) / (res_factor * d_a * d_b)
            self.ce[axis][sl[0], sl[1], sl[2]] = (2 * eps - dt * sig - sign * beta) / (
                2 * eps + dt * sig + beta)
            self.ceh_a[axis][sl[0], sl[1], sl[2]] = -2 * dt / ((2 * eps + dt * sig + beta) * d_b)
            self.ceh_b[axis][sl[0], sl[1], sl[2]] = 2 * dt / ((2 * eps + dt * sig + beta) * d_a)
            if kind == "current":
                amp = el.waveform.amplitude / (na * nb)
                if neg:
                    amp *= -1
                coff = -2 * dt / ((2 * eps + dt * sig + beta) * (d_b * d_a)) * amp
            elif kind == "voltage":
                amp = el.waveform.amplitude / nc
                if neg:
                    amp *= -1
                coff = -2 * dt / ((2 * eps + dt * sig + beta) * alpha) * amp
            else:
                continue
            self.lumped.append({"comp": axis, "s": s, "e": en,
                                "coff": np.ascontiguousarray(coff, dtype=np.float64),
                                "waveform": el.waveform})

    # ---------------------------------------------------------------- CPML
    def _pml(self):
        """PML::init/correctUpdateCoefficient/calRecursiveConvolutionCoeff
        (src/boundary/pml.cpp:98-196, 214-244, 286-633)."""
        self.pml = []
        nn = (self.nx, self.ny, self.nz)
        dt = self.dt
        for p in self.scene.pmls:
            m, neg = DIR[p.direction]
            n = abs(p.thickness)
            if neg:
                e_start, h_start = 1, 0
            else:
                e_start, h_start = nn[m] - n, nn[m] - n
            A, B = tan_a(m), tan_b(m)
            task_s = [0, 0, 0]
            task_e = list(nn)
            task_s[m], task_e[m] = h_start, h_start + n
            g_h = self.h_size[m][e_start:e_start + n]
            g_e = self.e_size[m][h_start:h_start + n]
            order = p.order

            def rho(size, frac):
                interval = size - frac * size
                d = np.zeros(n)
                d[0] = interval[0]
                total = 0.0
                for i in range(1, n):
                    total += size[i - 1]
                    d[i] = total + interval[i]
                total += size[n - 1]
                if neg:
                    d = d[::-1].copy()
                return d / total

            # C library pow/exp element by element, as xt::pow/xt::exp call them.
            cpow = lambda v: np.array([math.pow(x, order) for x in v.tolist()])
            cexp = lambda v: np.array([math.exp(x) for x in v.tolist()])
            sigma_max_e = p.sigma_ratio * (order + 1) / (150 * PI * float(np.min(g_h)))
            rho_e = rho(g_h, 0.75)
            sigma_e = sigma_max_e * cpow(rho_e)
            alpha_e = p.alpha_min + (p.alpha_max - p.alpha_min) * (1 - rho_e)
            kappa_e = 1 + (p.kappa_max - 1) * cpow(rho_e)
            b_e = cexp((-dt / EPSILON_0) * (sigma_e / kappa_e + alpha_e))
            a_e = (b_e - 1) * sigma_e / ((sigma_e + kappa_e * alpha_e) * kappa_e * g_h)
            e2m = MU_0 / EPSILON_0
            sigma_max_m = p.sigma_ratio * (order + 1) / (150 * PI * float(np.min(g_e))) * e2m
            rho_m = rho(g_e, 0.25)
            sigma_m = sigma_max_m * cpow(rho_m)
            alpha_m = (p.alpha_min + (p.alpha_max - p.alpha_min) * (1 - rho_m)) * e2m
            kappa_h = 1 + (p.kappa_max - 1) * cpow(rho_m)
            b_h = cexp((-dt / MU_0) * (sigma_m / kappa_h + alpha_m))
            a_h = (b_h - 1) * sigma_m / ((sigma_m + kappa_h * alpha_m) * kappa_h * g_e)
            # correctCoefficientX/Y/Z: the slab-normal curl coefficients
            # E_A<-H_B, E_B<-H_A, H_A<-E_B, H_B<-E_A.
            # E_A w.r.t. H_B is the "b" coefficient of E_A (H_B = tangential B of m is
            # tangential A or B of A?).  Resolve by axis: coefficient of E_c w.r.t. H_m.
            targets = [
                ("E", A, g_h, kappa_e, e_start),
                ("E", B, g_h, kappa_e, e_start),
                ("H", A, g_e, kappa_h, h_start),
                ("H", B, g_e, kappa_h, h_start),
            ]
            c_psi, psi = [], []
            shapes = []
            nloc = list(nn)
            nloc[m] = n
            for q, (kind, comp, dl, kap, start) in enumerate(targets):
                shp = list(nloc)
                if (kind == "E" and q == 0) or (kind == "H" and q == 3):
                    shp[B] += 1  # E_A / H_B: [A]=n_A, [B]=n_B+1
                else:
                    shp[A] += 1  # E_B / H_A: [A]=n_A+1, [B]=n_B
                shapes.append(tuple(shp))
                coeff = self._normal_coeff(kind, comp, m)
                sl = [slice(0, shp[0]), slice(0, shp[1]), slice(0, shp[2])]
                sl[m] = slice(start, start + n)
                view = coeff[tuple(sl)]
                bshape = [1, 1, 1]
                bshape[m] = n
                cp = np.ascontiguousarray(view * dl.reshape(bshape))
                coeff[tuple(sl)] = view / kap.reshape(bshape)
                c_psi.append(cp)
                psi.append(np.zeros(shp))
            self.pml.append({"m": m, "n": n, "e_start": e_start, "h_start": h_start,
                             "task_s": task_s, "task_e": task_e, "a_e": a_e, "b_e": b_e,
                             "a_h": a_h, "b_h": b_h, "c_psi": c_psi, "psi": psi,
                             "kappa_e": kappa_e, "kappa_h": kappa_h})

    def _normal_coeff(self, kind: str, comp: int, m: int) -> np.ndarray:
        """The coefficient of field `comp` w.r.t. the dual field along axis m's
        curl term, i.e. the slab-normal derivative coefficient."""
        A, B = tan_a(comp), tan_b(comp)
        # E_comp = ce E + ceh_a (dH_A/dB) + ceh_b (dH_B/dA); the term differencing
        # along m is ceh_a if m == B else ceh_b (m == A).
        if kind == "E":
            return self.ceh_a[comp] if m == B else self.ceh_b[comp]
        return self.che_a[comp] if m == B else self.che_b[comp]

    # ----------------------------------------------------------------- TFSF
    def _tfsf(self):
        """TFSF::defaultInit/initTransform/calculateProjection/
        initTimeDependentVariable (src/waveform_source/tfsf.cpp:14-340)."""
        t = self.scene.tfsf
        self.tfsf = None
        if t is None:
            return
        nn = (self.nx, self.ny, self.nz)
        org = (t.x, t.y, t.z)
        size = [nn[a] - 2 * org[a] for a in range(3)]
        st, ct = math.sin(t.theta), math.cos(t.theta)
        sp, cp = math.sin(t.phi), math.cos(t.phi)
        ss, cs = math.sin(t.psi), math.cos(t.psi)
        ratio = 1 / math.sqrt(math.pow(st, 4) * (math.pow(cp, 4) + math.pow(sp, 4)) +
                              math.pow(ct, 4))
        aux = int(math.ceil(ratio * math.sqrt(math.pow(size[0], 2) + math.pow(size[1], 2) +
                                              math.pow(size[2], 2)))) + 4 + 1
        k = np.array([st * cp, st * sp, ct])
        va = np.array([-sp, ct * cp, st * cp])
        vb = np.array([cp, ct * sp, st * sp])
        vc = np.array([0.0, -st, ct])
        ke = np.array([ss, cs, 0.0])
        te = np.array([va[0] * ke[0] + va[1] * ke[1] + va[2] * ke[2],
                       vb[0] * ke[0] + vb[1] * ke[1] + vb[2] * ke[2],
                       vc[0] * ke[0] + vc[1] * ke[1] + vc[2] * ke[2]])
        th = np.array([k[1] * te[2] - k[2] * te[1], k[2] * te[0] - k[0] * te[2],
                       k[0] * te[1] - k[1] * te[0]])
        # calculateInjectPostion (tfsf.cpp:304-340)
        inj = []
        for a in range(3):
            inj.append(org[a] if k[a] >= 0 else org[a] + size[a])
        extra = 2 * k / ratio
        inc = [inj[a] - extra[a] for a in range(3)]
        p_int, p_half = [], []
        for a in range(3):
            n_int = size[a] + 1
            p_int.append(np.array([((i + float(org[a])) - inc[a]) * k[a] * ratio
                                   for i in range(n_int)]))
            p_half.append(np.array([((i + float(org[a])) - inc[a] - 0.5) * k[a] * ratio
                                    for i in range(n_int + 1)]))
        scaled_dl = self.based[2] / ratio
        dt = self.dt
        ceie, chih = 1.0, 1.0
        ceih = -(dt / (EPSILON_0 * scaled_dl))
        chie = -(dt / (MU_0 * scaled_dl))
        abc0 = (C_0 * dt - scaled_dl) / (C_0 * dt + scaled_dl)
        abc1 = 2 * scaled_dl / (C_0 * dt + scaled_dl)
        nt = self.scene.steps
        e_time = linspace((0 + 1) * dt, (0 + nt) * dt, nt)
        source = t.waveform(e_time - dt)
        e_inc = np.zeros((nt, aux))
        h_inc = np.zeros((nt, aux - 1))
        nl = aux - 1
        # fdtd_1d (tfsf.cpp:40-68)
        e_inc[0, 0] = source[0]
        for l in range(1, nl):
            h_inc[0, l] = chih * h_inc[0, l] + chie * (e_inc[0, l + 1] - e_inc[0, l])
        for tt in range(1, nt):
            e_inc[tt, 0] = source[tt]
            e_inc[tt, 1:nl] = ceie * e_inc[tt - 1, 1:nl] + ceih * (h_inc[tt - 1, 1:nl] -
                                                                  h_inc[tt - 1, 0:nl - 1])
            ep2 = 0.0 if tt < 2 else e_inc[tt - 2, nl - 1]
            el2 = 0.0 if tt < 2 else e_inc[tt - 2, nl]
            e_inc[tt, nl] = (-ep2 + abc0 * (e_inc[tt, nl - 1] + el2) +
                             abc1 * (e_inc[tt - 1, nl] + e_inc[tt - 1, nl - 1]))
            h_inc[tt, 0:nl] = chih * h_inc[tt - 1, 0:nl] + chie * (e_inc[tt, 1:nl + 1] -
                                                                 e_inc[tt, 0:nl])
        ca = [dt / (EPSILON_0 * self.based[a]) for a in range(3)]
        cb = [dt / (MU_0 * self.based[a]) for a in range(3)]
        self.tfsf = {"box_s": list(org), "box_e": [org[a] + size[a] for a in range(3)],
                     "nt": nt, "aux": aux, "e_inc": e_inc, "h_inc": h_inc,
                     "p_int": p_int, "p_half": p_half, "ca": ca, "cb": cb, "te": te,
                     "th": th, "source": source, "ratio": ratio, "k": k}

    # ------------------------------------------------------------------ ADE
    def _ade(self):
        """Simulation::buildDispersiveSpace (simulation.cpp:745-829),
        Object::handleDispersion (object.cpp:52-98), the three
        ADEMethodStorage::correctCoeff variants and makeUpdator (:688-743)."""
        self.ade = None
        disp = [m for m in self.materials if m.dispersive]
        if not disp:
            return
        num_pole = max(len(m.poles) for m in disp)
        kinds = {m.kind for m in disp}
        if kinds == {"drude"}:
            kind = 1
        elif kinds == {"debye"}:
            kind = 2
        else:
            kind = 0
        nx, ny, nz = self.nx, self.ny, self.nz
        shp4 = (nx, ny, nz, num_pole)
        shp3 = (nx, ny, nz)
        z4 = lambda: np.zeros(shp4)
        st = {"kind": kind, "np": num_pole, "cjj": z4(), "cje": z4(), "cjsumj": z4(),
              "cejsum": np.zeros(shp3), "j": [z4() for _ in range(3)]}
        if kind == 0:
            st.update({"cjjp": z4(), "cjen": z4(), "cjep": z4(), "cjsumjp": z4(),
                       "ceep": np.zeros(shp3), "eprev": [np.zeros(shp3) for _ in range(3)],
                       "jprev": [z4() for _ in range(3)]})
        dt = self.dt
        hx, hy, hz = self.h_size
        for index, mat in enumerate(self.materials):
            if not mat.dispersive:
                continue
            cells = np.argwhere(self.cell_material == index)
            if cells.size == 0:
                continue
            P = len(mat.poles)
            if kind == 0:
                a0, a1, b0, b1, b2 = self._mlorentz_params(mat)
                a = (a1 * EPSILON_0 / (dt * dt)) + (0.5 * a0 * EPSILON_0 / dt)
                b = (-2 * a1 * EPSILON_0) / (dt * dt)
                c = (a1 * EPSILON_0 / (dt * dt)) - (0.5 * a0 * EPSILON_0 / dt)
                d = (2 * b2 / (dt * dt)) - b0
                e = (-b2 / (dt * dt)) + (b1 / (2 * dt))
                f = (b2 / (dt * dt)) + (b1 / (2 * dt))
                sum_a_f = 0.0
                sum_b_f = 0.0
                sum_c_f = 0.0
                for p in range(P):
                    sum_a_f += a[p] / f[p]
                for p in range(P):
                    sum_b_f += b[p] / f[p]
                for p in range(P):
                    sum_c_f += c[p] / f[p]
                sigma_e = SIGMA_E_ZERO
                temp = (mat.eps_inf * EPSILON_0) / dt + 0.5 * sum_a_f + 0.5 * sigma_e
                cece = ((mat.eps_inf * EPSILON_0) / dt - 0.5 * sum_b_f - 0.5 * sigma_e) / temp
                i, j, k_ = cells[:, 0], cells[:, 1], cells[:, 2]
                for p in range(P):
                    st["cjen"][i, j, k_, p] = a[p] / f[p]
                    st["cje"][i, j, k_, p] = b[p] / f[p]
                    st["cjep"][i, j, k_, p] = c[p] / f[p]
                    st["cjj"][i, j, k_, p] = d[p] / f[p]
                    st["cjjp"][i, j, k_, p] = e[p] / f[p]
                    st["cjsumj"][i, j, k_, p] = 0.5 * (1 + d[p] / f[p])
                    st["cjsumjp"][i, j, k_, p] = 0.5 * (e[p] / f[p])
                st["cejsum"][i, j, k_] = -1 / temp
                st["ceep"][i, j, k_] = -0.5 * sum_c_f / temp
                dx, dy, dz = hx[i], hy[j], hz[k_]
                self._ade_overwrite(i, j, k_, dx, dy, dz, lambda db: -1 / (temp * db),
                                    lambda da: 1 / (temp * da), cece)
            else:
                sigma = SIGMA_E_ZERO
                if kind == 1:
                    wp = np.array([p_[0] for p_ in mat.poles])
                    gm = np.array([p_[1] for p_ in mat.poles])
                    kk = (1 - gm * dt / 2) / (1 + gm * dt / 2)
                    beta = (EPSILON_0 * wp * wp * dt / 2) / (1 + gm * dt / 2)
                    sum_beta = 0.0
                    for v in beta:
                        sum_beta += v
                    ca_ = (2 * EPSILON_0 * mat.eps_inf - dt * sum_beta - dt * sigma) / (
                        2 * EPSILON_0 * mat.eps_inf - dt * sum_beta + dt * sigma)
                    cb_ = (2 * dt) / (2 * EPSILON_0 * mat.eps_inf - dt * sum_beta + dt * sigma)
                    cje = beta
                else:
                    es_ = np.array([p_[0] for p_ in mat.poles])
                    tau = np.array([p_[1] for p_ in mat.poles])
                    de = es_ - mat.eps_inf
                    kk = (2 * tau - dt) / (2 * tau + dt)
                    beta = (2 * EPSILON_0 * de * dt) / (2 * tau + dt)
                    sum_beta = 0.0
                    for v in beta:
                        sum_beta += v
                    ca_ = (2 * EPSILON_0 * mat.eps_inf + sum_beta - dt * sigma) / (
                        2 * EPSILON_0 * mat.eps_inf + sum_beta + dt * sigma)
                    cb_ = (2 * dt) / (2 * EPSILON_0 * mat.eps_inf + sum_beta + dt * sigma)
                    cje = beta / dt
                i, j, k_ = cells[:, 0], cells[:, 1], cells[:, 2]
                # Pole loop runs to the storage's pole count (drude_ade_method.cpp:115-119).
                for p in range(P):
                    st["cjj"][i, j, k_, p] = kk[p]
                    st["cje"][i, j, k_, p] = cje[p]
                    st["cjsumj"][i, j, k_, p] = 0.5 * (1 + kk[p])
                st["cejsum"][i, j, k_] = -cb_
                dx, dy, dz = hx[i], hy[j], hz[k_]
                self._ade_overwrite(i, j, k_, dx, dy, dz, lambda db: -cb_ / db,
                                    lambda da: cb_ / da, ca_)
        self.ade = st

    @staticmethod
    def _mlorentz_params(mat):
        """MLorentz (a0, a1, b0, b1, b2) of each pole; Drude and Debye map onto
        it as DrudeEqDecision / DebyeEqDecision do
        (src/material/dispersive_material_equation.cpp:43-54)."""
        P = len(mat.poles)
        if mat.kind == "mlorentz":
            arr = np.array(mat.poles, dtype=np.float64).reshape(P, 5)
            return arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3], arr[:, 4]
        if mat.kind == "drude":
            wp = np.array([p[0] for p in mat.poles])
            gm = np.array([p[1] for p in mat.poles])
            return wp * wp, np.zeros(P), np.zeros(P), gm, np.ones(P)
        es_ = np.array([p[0] for p in mat.poles])
        tau = np.array([p[1] for p in mat.poles])
        return es_ - mat.eps_inf, np.zeros(P), np.ones(P), tau, np.zeros(P)

    def _ade_overwrite(self, i, j, k, dx, dy, dz, f_cha, f_chb, cece):
        """correct_func of the ADE storages: cece, cecha = f(db), cechb = f(da)
        with (da, db) = (dy, dz) for Ex, (dz, dx) for Ey, (dx, dy) for Ez."""
        pairs = [(dy, dz), (dz, dx), (dx, dy)]
        for c in range(3):
            da, db = pairs[c]
            self.ce[c][i, j, k] = cece
            self.ceh_a[c][i, j, k] = f_cha(db)
            self.ceh_b[c][i, j, k] = f_chb(da)

    # ---------------------------------------------------------------- NF2FF
    def _huygens_tasks(self, d):
        """NFFFT::initGlobal/makeNodeAxisTask (src/nffft/nffft.cpp:88-245), one
        domain: per face XN..ZP ([s], [e]) or None."""
        nn = (self.nx, self.ny, self.nz)
        gs = [d[a] for a in range(3)]
        ge = [nn[a] - d[a] for a in range(3)]
        tasks = []
        for face in range(6):
            m, positive = face // 2, face % 2
            s = list(gs)
            e = list(ge)
            c = ge[m] if positive else gs[m]
            if (not positive) and (c <= 0 or c == 1):
                tasks.append(None)
                continue
            if positive and c >= nn[m]:
                tasks.append(None)
                continue
            s[m], e[m] = c, c + 1
            for a in range(3):  # make_secondary_axis_range
                if a == m:
                    continue
                if s[a] <= 0:
                    s[a] = 1
                if e[a] >= nn[a]:
                    e[a] = nn[a] - 1
            tasks.append((s, e))
        return tasks

    def _nf2ff_td(self):
        """NFFFTTimeDomain::initTimeDependentVariable and distanceRange
        (src/nffft/nfffft_time_domain.cpp:49-78, 414-479), the per-point delay
        and face-cell area of TDPlaneData (src/include/nffft/nffft_td_data.h:
        22-46, 338-362)."""
        self.nf2ff_td = None
        spec = getattr(self.scene, "nf2ff_td", None)
        if spec is None:
            return
        tasks = self._huygens_tasks(spec.distance)
        ru = (math.sin(spec.theta) * math.cos(spec.phi), math.sin(spec.theta) * math.sin(spec.phi),
              math.cos(spec.theta))
        proj, ds = [], []
        for face, task in enumerate(tasks):
            if task is None:
                continue
            s, e = task
            m = face // 2
            A, B = (m + 1) % 3, (m + 2) % 3
            axes = [self.e_node[a] if a == m else self.h_node[a] for a in range(3)]
            R = np.meshgrid(*[axes[a][s[a]:e[a]] for a in range(3)], indexing="ij")
            proj.append((R[0] * ru[0] + R[1] * ru[1] + R[2] * ru[2]).ravel())
            sz = [self.e_size[a][s[a]:e[a]] for a in range(3)]
            S = np.meshgrid(*sz, indexing="ij")
            ds.append((S[A] * S[B]).ravel())
        if not proj:
            return
        proj = np.concatenate(proj)
        ds = np.ascontiguousarray(np.concatenate(ds))
        lo, hi = float(proj.min()), float(proj.max())
        dt = self.dt
        delay = np.ascontiguousarray((hi - proj) / (C_0 * dt))
        n_bins = int(math.ceil((hi - lo) / (C_0 * dt))) + self.scene.steps + 4
        P = proj.size
        self.nf2ff_td = {"tasks": tasks, "delay": delay, "ds": ds, "P": P, "n_bins": n_bins,
                         "prev": np.zeros(4 * P), "pot": np.zeros(6 * 4 * n_bins),
                         "theta": spec.theta, "phi": spec.phi}

    def nf2ff_td_far_field(self) -> Dict[str, np.ndarray]:
        """NFFFTTimeDomain::wx..uz and processFarField
        (src/nffft/nfffft_time_domain.cpp:98-160, 481-509): w_theta, w_phi,
        u_theta, u_phi over the retarded-time bins."""
        td = self.nf2ff_td
        nb = td["n_bins"]
        pot = td["pot"].reshape(6, 4, nb)
        den = C_0 * self.dt * 4 * PI
        ua, ub, wa, wb = (pot[:, q] / den for q in range(4))
        XN, XP, YN, YP, ZN, ZP = range(6)
        wx = wa[ZN] + wa[ZP] + wb[YN] + wb[YP]
        wy = wa[XN] + wa[XP] + wb[ZN] + wb[ZP]
        wz = wb[XN] + wb[XP] + wa[YN] + wa[YP]
        ux = ua[ZN] + ua[ZP] + ub[YN] + ub[YP]
        uy = ua[XN] + ua[XP] + ub[ZN] + ub[ZP]
        uz = ub[XN] + ub[XP] + ua[YN] + ua[YP]
        ct, st = math.cos(td["theta"]), math.sin(td["theta"])
        cp, sp = math.cos(td["phi"]), math.sin(td["phi"])
        return {"w_theta": wx * ct * cp + wy * ct * sp - wz * st, "w_phi": -wx * sp + wy * cp,
                "u_theta": ux * ct * cp + uy * ct * sp - uz * st, "u_phi": -ux * sp + uy * cp}

    def _nf2ff(self):
        """NFFFT::initGlobal/makeNodeAxisTask (src/nffft/nffft.cpp:88-245) and
        FDPlaneData::initDFT (src/nffft/nffft_fd_data.cpp:65-76)."""
        self.nf2ff = None
        spec = self.scene.nf2ff
        if spec is None:
            return
        nn = (self.nx, self.ny, self.nz)
        d = spec.distance
        gs = [d[a] for a in range(3)]
        ge = [nn[a] - d[a] for a in range(3)]
        tasks = []
        for face in range(6):
            m, positive = face // 2, face % 2
            s = list(gs)
            e = list(ge)
            c = ge[m] if positive else gs[m]
            if (not positive) and (c <= 0 or c == 1):
                tasks.append(None)
                continue
            if positive and c >= nn[m]:
                tasks.append(None)
                continue
            s[m], e[m] = c, c + 1
            for a in range(3):  # make_secondary_axis_range
                if a == m:
                    continue
                if s[a] <= 0:
                    s[a] = 1
                if e[a] >= nn[a]:
                    e[a] = nn[a] - 1
            tasks.append((s, e))
        nf = len(spec.freqs)
        nt = self.scene.steps
        dt = self.dt
        te = np.zeros((nf, nt, 2))
        th = np.zeros((nf, nt, 2))
        for fi, f in enumerate(spec.freqs):
            for t in range(nt):
                # dt * std::exp(-j 2 pi f (t+1) dt): the C library cos/sin of the angle
                ae = (-2.0 * PI) * ((f * (t + 1)) * dt)
                ah = (-2.0 * PI) * ((f * (t + 0.5)) * dt)
                te[fi, t, 0] = dt * math.cos(ae)
                te[fi, t, 1] = dt * math.sin(ae)
                th[fi, t, 0] = dt * math.cos(ah)
                th[fi, t, 1] = dt * math.sin(ah)
        offs = []
        total = 0
        for fi in range(nf):
            for face in range(6):
                npts = 0
                if tasks[face] is not None:
                    s, e = tasks[face]
                    npts = (e[0] - s[0]) * (e[1] - s[1]) * (e[2] - s[2])
                for q in range(4):
                    offs.append(total)
                    total += npts
        self.nf2ff = {"nf": nf, "nt": nt, "tasks": tasks, "te": te, "th": th,
                      "acc": np.zeros(2 * total), "off": np.array(offs, dtype=np.int64),
                      "freqs": np.array(spec.freqs, dtype=np.float64)}

    def far_field(self, theta, phi, origin=(0.0, 0.0, 0.0)) -> np.ndarray:
        """Far-field potentials from the accumulated surface currents:
        FDPlaneData::getPotential / calculatePotential
        (src/nffft/nffft_fd_data_process.cpp:15-144) summed over the faces
        XN, XP, YN, YP, ZN, ZP, for every frequency in the order of
        NFFFTFrequencyDomain::processFarField
        (src/nffft/nffft_frequency_domain.cpp:103-129): returns complex
        [n_freq, 4, n_angles] with rows a_theta, f_phi, a_phi, f_theta.
        Face-centre positions rVector and areas ds follow
        nffft_fd_data_process.cpp:185-215; the Cartesian-to-spherical unit
        vector components follow cCSToSCSTransformMatrix
        (include/xfdtd/util/transform.h:25-59)."""
        theta = np.atleast_1d(np.asarray(theta, dtype=np.float64))
        phi = np.atleast_1d(np.asarray(phi, dtype=np.float64))
        if theta.size != 1 and phi.size != 1:
            raise ValueError("There must be only one theta or phi")
        n_ang = theta.size * phi.size
        th = np.broadcast_to(theta, (n_ang,)) if theta.size == n_ang else np.full(n_ang, theta[0])
        ph = np.broadcast_to(phi, (n_ang,)) if phi.size == n_ang else np.full(n_ang, phi[0])
        cos_t, sin_t = np.cos(th), np.sin(th)
        cos_p, sin_p = np.cos(ph), np.sin(ph)
        st_sp, st_cp = sin_t * sin_p, sin_t * cos_p
        # unit vectors of the Cartesian axes projected on theta-hat / phi-hat
        tr = {"theta": [cos_t * cos_p, cos_t * sin_p, -1 * sin_t],
              "phi": [-1 * sin_p, cos_p, np.zeros_like(th)]}
        nf = self.nf2ff
        out = np.zeros((nf["nf"], 4, n_ang), dtype=np.complex128)
        plan = [(0, "theta"), (2, "phi"), (0, "phi"), (2, "theta")]  # (q of a, scs)
        for fi, freq in enumerate(nf["freqs"]):
            k0 = 2.0 * PI * freq / C_0
            for row, (q0, scs) in enumerate(plan):
                acc = np.zeros(n_ang, dtype=np.complex128)
                for face in range(6):
                    if nf["tasks"][face] is None:
                        continue
                    s, e = nf["tasks"][face]
                    m = face // 2
                    A, B = (m + 1) % 3, (m + 2) % 3
                    a = self.nf2ff_surface(fi, face, q0).ravel()
                    b = self.nf2ff_surface(fi, face, q0 + 1).ravel()
                    ii, jj, kk = np.meshgrid(np.arange(s[0], e[0]), np.arange(s[1], e[1]),
                                             np.arange(s[2], e[2]), indexing="ij")
                    idx = [ii.ravel(), jj.ravel(), kk.ravel()]
                    pos = [(self.e_node[x] if x == m else self.h_node[x])[idx[x]] - origin[x]
                           for x in range(3)]
                    ds = self.e_size[A][idx[A]] * self.e_size[B][idx[B]]
                    arg = (pos[0][:, None] * st_cp[None, :] + pos[1][:, None] * st_sp[None, :]
                           + pos[2][:, None] * cos_t[None, :])
                    phase = np.exp(1j * k0 * arg)
                    term = (a[:, None] * tr[scs][A][None, :] + b[:, None] * tr[scs][B][None, :])
                    acc += np.sum(term * phase * ds[:, None], axis=0)
                out[fi, row] = acc
        return out

    def radiation_power(self) -> np.ndarray:
        """Radiated power per frequency: FDPlaneData::power / calculatePower
        (src/nffft/nffft_fd_data_process.cpp:38-190), 0.5 Re of the sum over
        the faces XN..ZP of (-1 on the negative faces) sum ds (conj(J_a) M_b -
        conj(J_b) M_a), ds the E-cell sizes across the face."""
        nf = self.nf2ff
        out = np.zeros(nf["nf"])
        for fi in range(nf["nf"]):
            total = 0j
            for face in range(6):
                if nf["tasks"][face] is None:
                    continue
                s, e = nf["tasks"][face]
                m = face // 2
                A, B = (m + 1) % 3, (m + 2) % 3
                ja, jb, ma, mb = (self.nf2ff_surface(fi, face, q).ravel() for q in range(4))
                ii, jj, kk = np.meshgrid(np.arange(s[0], e[0]), np.arange(s[1], e[1]),
                                         np.arange(s[2], e[2]), indexing="ij")
                idx = [ii.ravel(), jj.ravel(), kk.ravel()]
                ds = self.e_size[A][idx[A]] * self.e_size[B][idx[B]]
                acc = np.sum(ds * (np.conj(ja) * mb - np.conj(jb) * ma))
                total += (-1.0 if face % 2 == 0 else 1.0) * acc
            out[fi] = 0.5 * total.real
        return out

    def nf2ff_surface(self, f: int, face: int, q: int) -> Optional[np.ndarray]:
        """Complex accumulator (ja, jb, ma, mb) of frequency f on face d, shaped
        like the face task."""
        nf = self.nf2ff
        task = nf["tasks"][face]
        if task is None:
            return None
        s, e = task
        shape = tuple(e[a] - s[a] for a in range(3))
        npts = shape[0] * shape[1] * shape[2]
        o = int(nf["off"][(f * 6 + face) * 4 + q])
        flat = nf["acc"][2 * o:2 * (o + npts)]
        return (flat[0::2] + 1j * flat[1::2]).reshape(shape)

    # ------------------------------------------------------------- monitors
    def _monitors(self):
        """FieldMonitor::init box with the +1 origin shift at index 0
        (src/monitor/field_monitor.cpp:17-67); MovieMonitor::update
        (src/monitor/movie_monitor.cpp:26-34)."""
        self.movies = []
        for mv in self.scene.movies:
            o, e = self.grid_box(mv.shape)
            o = list(o)
            size = [e[a] - o[a] for a in range(3)]
            for a in range(3):
                if o[a] == 0:
                    o[a] += 1
                    size[a] -= 1
            self.movies.append({"name": mv.name, "field": mv.field, "interval": mv.interval,
                                "s": o, "e": [o[a] + size[a] for a in range(3)], "count": 0})
            self.movie_frames[mv.name] = []
        # FieldTimeMonitor::init/update (src/monitor/field_time_monitor.cpp:17-95):
        # the same box shift; update() overwrites data(t) for every node of the
        # box, leaving the value of its last node.
        self.field_times = []
        self.field_time_data: Dict[str, np.ndarray] = {}
        nt = self.scene.steps
        for ft in self.scene.field_times:
            o, e = self.grid_box(ft.shape)
            o = list(o)
            size = [e[a] - o[a] for a in range(3)]
            for a in range(3):
                if o[a] == 0:
                    o[a] += 1
                    size[a] -= 1
            last = None
            if all(size[a] > 0 for a in range(3)):
                last = [o[a] + size[a] - 1 for a in range(3)]
            self.field_times.append({"name": ft.name, "field": ft.field, "node": last})
            t_arr = (linspace((0 + 1) * self.dt, (0 + nt) * self.dt, nt) if ft.field[0] == "E"
                     else linspace((0 + 0.5) * self.dt, (0 + nt + 0.5) * self.dt, nt))
            self.field_time_data[ft.name] = np.stack([t_arr, np.zeros(nt)])
        self._line_monitors()

    def _line_monitors(self):
        """VoltageMonitor::init/update (src/monitor/voltage_monitor.cpp:17-235)
        and CurrentMonitor::init/update (src/monitor/current_monitor.cpp:17-379)
        for one domain (node task = global task, lower corner 0, upper corner
        n), as lists of (field name, node, weight) summed every step."""
        self.line_monitors = []
        self.line_monitor_data: Dict[str, np.ndarray] = {}
        nt = self.scene.steps
        n = (self.nx, self.ny, self.nz)
        for spec in getattr(self.scene, "line_monitors", []):
            c = "XYZ".index(spec.direction[0])
            neg = spec.direction[1] == "N"
            a, b = (c + 1) % 3, (c + 2) % 3
            o, e = self.grid_box(spec.shape)
            entries = []
            if spec.kind == "voltage":
                r = [None, None, None]
                for ax in (a, b):
                    s0, s1 = o[ax], e[ax] + 1
                    if s0 <= 0:
                        s0 = 1
                    if n[ax] <= s1:
                        s1 = n[ax] - 1
                    r[ax] = (s0, s1)
                r[c] = (o[c], e[c])
                if any(r[q][1] <= r[q][0] for q in range(3)):
                    raise ValueError(f"{spec.name} globalTask is not valid")
                nab = (r[a][1] - r[a][0]) * (r[b][1] - r[b][0])
                for i in range(*r[0]):
                    for j in range(*r[1]):
                        for k in range(*r[2]):
                            x = (i, j, k)
                            coff = -self.h_size[c][x[c]] / float(nab)
                            if neg:
                                coff *= -1.0
                            entries.append(("E" + "XYZ"[c], x, coff))
                t_arr = linspace((0 + 1) * self.dt, (0 + nt) * self.dt, nt)
            else:
                if e[c] == 0 or o[a] == 0 or e[a] == n[a] or o[b] == 0 or e[b] == n[b]:
                    raise ValueError(f"{spec.name}: invalid current monitor box")
                lo, hi = list(o), list(e)
                lo[c] = e[c] - 1

                def ranges(b_start, b_end, n_b, n_a, start, end):
                    if start <= 0:
                        start = 1
                    end = end + 1
                    if n_a <= end:
                        end = n_a - 1
                    rn = (start, end) if b_start not in (0, n_b - 1, n_b) else (0, 0)
                    rp = (start, end) if b_end not in (n_b, n_b - 1, 0) else (0, 0)
                    return rn, rp

                ha_bn, ha_bp = ranges(lo[b], hi[b], n[b], n[a], lo[a], hi[a])
                hb_an, hb_ap = ranges(lo[a], hi[a], n[a], n[b], lo[b], hi[b])
                sgn = -1.0 if neg else 1.0
                plane = hi[c] - 1

                def node(av, bv):
                    x = [0, 0, 0]
                    x[a], x[b], x[c] = av, bv, plane
                    return tuple(x)

                for v in range(*ha_bn):
                    entries.append(("H" + "XYZ"[a], node(v, lo[b] - 1), sgn * self.e_size[a][v]))
                for v in range(*ha_bp):
                    entries.append(("H" + "XYZ"[a], node(v, hi[b]), -sgn * self.e_size[a][v]))
                for v in range(*hb_an):
                    entries.append(("H" + "XYZ"[b], node(lo[a] - 1, v), -sgn * self.e_size[b][v]))
                for v in range(*hb_ap):
                    entries.append(("H" + "XYZ"[b], node(hi[a], v), sgn * self.e_size[b][v]))
                t_arr = linspace((0 + 0.5) * self.dt, (0 + nt + 0.5) * self.dt, nt)
            self.line_monitors.append({"name": spec.name, "entries": entries})
            self.line_monitor_data[spec.name] = np.stack([t_arr, np.zeros(nt)])

    # ----------------------------------------------------------------- init
    def _init(self):
        self._grid()
        nx, ny, nz = self.nx, self.ny, self.nz
        # Simulation::generateEMF (simulation.cpp:514-528)
        self.e = [np.zeros((nx, ny + 1, nz + 1)), np.zeros((nx + 1, ny, nz + 1)),
                  np.zeros((nx + 1, ny + 1, nz))]
        self.h = [np.zeros((nx + 1, ny, nz)), np.zeros((nx, ny + 1, nz)),
                  np.zeros((nx, ny, nz + 1))]
        self._materials()
        self._coefficients()
        # Simulation::correctUpdateCoefficient (simulation.cpp:638-652):
        # objects (thin wires, lumped) -> boundaries (PML) -> sources ->
        # dispersive space.
        self._thin_wires()
        self._current_sources()
        self._pml()
        self._tfsf()
        self._ade()
        self._nf2ff()
        self._nf2ff_td()
        self._monitors()
        nt = self.scene.steps
        h_time = linspace((0 + 0.5) * self.dt, (0 + nt + 0.5) * self.dt, nt)
        for l in self.lumped:  # CurrentSource / VoltageSource ::initTimeDependentVariable
            if "waveform" in l:
                l["wave"] = np.ascontiguousarray(l["waveform"](h_time))
        self._bind()
        self.t = 0

    def _bind(self):
        k = self._keep
        y = _Yee()
        y.nx, y.ny, y.nz = self.nx, self.ny, self.nz
        for c in range(3):
            y.e[c] = _arr(self.e[c])
            y.h[c] = _arr(self.h[c])
            y.ce[c] = _arr(self.ce[c])
            y.ceh_a[c] = _arr(self.ceh_a[c])
            y.ceh_b[c] = _arr(self.ceh_b[c])
            y.ch[c] = _arr(self.ch[c])
            y.che_a[c] = _arr(self.che_a[c])
            y.che_b[c] = _arr(self.che_b[c])
        k.append(y)
        sim = _Sim()
        sim.yee = ctypes.pointer(y)
        if self.ade is not None:
            a = _Ade()
            st = self.ade
            a.kind, a.np = st["kind"], st["np"]
            for name in ("cjj", "cjjp", "cjen", "cje", "cjep", "cjsumj", "cjsumjp", "cejsum",
                         "ceep"):
                setattr(a, name, _ptr(st.get(name)))
            for c in range(3):
                a.j[c] = _ptr(st["j"][c])
                if st["kind"] == 0:
                    a.eprev[c] = _ptr(st["eprev"][c])
                    a.jprev[c] = _ptr(st["jprev"][c])
            k.append(a)
            sim.ade = ctypes.pointer(a)
        pmls = (_Pml * max(1, len(self.pml)))()
        for i, p in enumerate(self.pml):
            s = pmls[i]
            s.m, s.n, s.e_start, s.h_start = p["m"], p["n"], p["e_start"], p["h_start"]
            for d in range(3):
                s.task_s[d], s.task_e[d] = p["task_s"][d], p["task_e"][d]
            s.a_e, s.b_e, s.a_h, s.b_h = (_ptr(p["a_e"]), _ptr(p["b_e"]), _ptr(p["a_h"]),
                                          _ptr(p["b_h"]))
            for q in range(4):
                s.c_psi[q] = _arr(p["c_psi"][q])
                s.psi[q] = _arr(p["psi"][q])
        k.append(pmls)
        sim.pml = ctypes.cast(pmls, ctypes.POINTER(_Pml))
        sim.n_pml = len(self.pml)
        if self.tfsf is not None:
            t = self.tfsf
            s = _Tfsf()
            s.is_, s.js, s.ks = t["box_s"]
            s.ie, s.je, s.ke = t["box_e"]
            s.nt, s.aux = t["nt"], t["aux"]
            # an x-slab of a decomposed lattice: box indices global, the slab
            # from global plane x_offset (tfsf_3d.cpp:21-33 cuts by domain)
            s.xo, s.nxl = int(t.get("x_offset", 0)), self.nx
            s.e_inc, s.h_inc = _ptr(t["e_inc"]), _ptr(t["h_inc"])
            for a in range(3):
                s.p_int[a] = _ptr(t["p_int"][a])
                s.p_half[a] = _ptr(t["p_half"][a])
                s.ca[a], s.cb[a] = t["ca"][a], t["cb"][a]
                s.te[a], s.th[a] = t["te"][a], t["th"][a]
            k.append(s)
            sim.tfsf = ctypes.pointer(s)
        lums = (_Lumped * max(1, len(self.lumped)))()
        for i, l in enumerate(self.lumped):
            s = lums[i]
            s.comp = l["comp"]
            for d in range(3):
                s.s[d], s.e[d] = l["s"][d], l["e"][d]
            s.coff = _ptr(l["coff"])
            if "j" in l:
                s.cecjc, s.j = _ptr(l["cecjc"]), _ptr(l["j"])
            else:
                s.wave = _ptr(l["wave"])
        k.append(lums)
        sim.lumped = ctypes.cast(lums, ctypes.POINTER(_Lumped))
        sim.n_lumped = len(self.lumped)
        if self.nf2ff is not None:
            nf = self.nf2ff
            s = _Nf2ff()
            s.nf, s.nt = nf["nf"], nf["nt"]
            for face in range(6):
                task = nf["tasks"][face]
                for d in range(3):
                    if task is None:
                        s.task_s[face][d], s.task_e[face][d] = 0, 0
                    else:
                        s.task_s[face][d], s.task_e[face][d] = task[0][d], task[1][d]
            s.te, s.th = _ptr(nf["te"]), _ptr(nf["th"])
            s.acc = _ptr(nf["acc"])
            s.off = nf["off"].ctypes.data_as(ctypes.POINTER(_i64))
            k.append(s)
            sim.nf2ff = ctypes.pointer(s)
        if self.nf2ff_td is not None:
            td = self.nf2ff_td
            s = _Nf2ffTd()
            for face in range(6):
                task = td["tasks"][face]
                for d in range(3):
                    if task is None:
                        s.task_s[face][d], s.task_e[face][d] = 0, 0
                    else:
                        s.task_s[face][d], s.task_e[face][d] = task[0][d], task[1][d]
            s.delay, s.ds = _ptr(td["delay"]), _ptr(td["ds"])
            s.prev, s.pot = _ptr(td["prev"]), _ptr(td["pot"])
            s.P, s.n_bins = td["P"], td["n_bins"]
            k.append(s)
            sim.nf2ff_td = ctypes.pointer(s)
        k.append(sim)
        self._sim = sim

    # ------------------------------------------------------------------ run
    def _record_monitors(self):
        for lm in self.line_monitors:
            v = 0.0
            for fname, x, w in lm["entries"]:
                arr = (self.e if fname[0] == "E" else self.h)["XYZ".index(fname[1])]
                v += w * arr[x]
            self.line_monitor_data[lm["name"]][1, self.t] = v
        for ft in self.field_times:
            if ft["node"] is not None:
                f = ft["field"]
                arr = (self.e if f[0] == "E" else self.h)["XYZ".index(f[1])]
                self.field_time_data[ft["name"]][1, self.t] = arr[tuple(ft["node"])]
        for mv in self.movies:
            if mv["count"] % mv["interval"] == 0:
                f = mv["field"]
                arr = (self.e if f[0] == "E" else self.h)["XYZ".index(f[1])]
                s, e = mv["s"], mv["e"]
                self.movie_frames[mv["name"]].append(
                    arr[s[0]:e[0], s[1]:e[1], s[2]:e[2]].copy())
            mv["count"] += 1

    def run(self, nsteps: Optional[int] = None):
        L = lib()
        if self.threads:
            L.orc_set_num_threads(self.threads)
        n = self.scene.steps - self.t if nsteps is None else nsteps
        if not self.movies and not getattr(self, "field_times", None) and \
                not getattr(self, "line_monitors", None):
            L.orc_run(ctypes.byref(self._sim), self.t, n)
            self.t += n
            return
        for _ in range(n):
            L.orc_step(ctypes.byref(self._sim), self.t)
            self._record_monitors()
            self.t += 1

    # -------------------------------------------------------------- outputs
    def fields(self) -> Dict[str, np.ndarray]:
        return {"EX": self.e[0], "EY": self.e[1], "EZ": self.e[2], "HX": self.h[0],
                "HY": self.h[1], "HZ": self.h[2]}


def network_s_parameters(sim: "RefSimulation", network) -> Dict[int, np.ndarray]:
    """Network::output's S-parameters (src/network/network.cpp:47-65) from the
    ports' waves (Port::calculateSParameters, src/network/port.cpp:104-130)
    and the reference's DFT (include/xfdtd/util/dft.h:9-26):
    X(f) = dt sum_n x_n exp(-j 2 pi f ((n + 1) dt + shift)), shift -1.5 dt for
    the current.  Keys are 10 j + i for source port i."""
    dt = sim.dt
    f = np.asarray(network.frequencies, dtype=np.float64)

    def dft(x, shift):
        t = (np.arange(len(x)) + 1) * dt + shift
        return dt * (x[None, :] * np.exp(-2j * np.pi * f[:, None] * t[None, :])).sum(axis=1)

    waves = {}
    for p in network.ports:
        i = dft(sim.line_monitor_data[p.current][1], -1.5 * dt)
        v = dft(sim.line_monitor_data[p.voltage][1], 0.0)
        z = complex(p.impedance)
        k = np.sqrt(z.real)
        waves[p.index] = (0.5 * (v + z * i) / k, 0.5 * (v - np.conj(z) * i) / k)
    out = {}
    for pi in network.ports:
        if not pi.is_source:
            continue
        for pj in network.ports:
            out[pj.index * 10 + pi.index] = waves[pj.index][1] / waves[pi.index][0]
    return out
