"""ctypes binding of the engine C ABI (include/xfd_engine.h).

This is the Python side of the drop-in boundary: every call goes through
``lib/libxfd_engine.so``; there is no Python or CPU implementation of the
time step behind it.  If the library is missing, or no CUDA device is
present, the calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import build as _build

FP64, FP32 = 0, 1
FIELD_NAMES = ("EX", "EY", "EZ", "HX", "HY", "HZ")
_STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "UNSUPPORTED", 4: "STATE",
           5: "OUT_OF_MEMORY", 6: "NUMERIC", 7: "TIMEOUT"}

_dp = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


class GridDesc(ctypes.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("precision", _i32),
                ("n_steps", _i64), ("dt", ctypes.c_double), ("device", _i32)]


class CpmlSlab(ctypes.Structure):
    _fields_ = [("axis", _i32), ("negative", _i32), ("thickness", _i32), ("e_start", _i32),
                ("h_start", _i32), ("a_e", _dp), ("b_e", _dp), ("a_h", _dp), ("b_h", _dp)]


class TfsfDesc(ctypes.Structure):
    _fields_ = [("box_s", _i32 * 3), ("box_e", _i32 * 3), ("aux", _i32), ("e_inc", _dp),
                ("h_inc", _dp), ("p_int", _dp * 3), ("p_half", _dp * 3),
                ("ca", ctypes.c_double * 3), ("cb", ctypes.c_double * 3),
                ("te", ctypes.c_double * 3), ("th", ctypes.c_double * 3)]


class AdeDesc(ctypes.Structure):
    _fields_ = [("kind", _i32), ("n_poles", _i32), ("n_materials", _i32), ("mat_coeff", _dp),
                ("n_entries", _i64), ("comp", ctypes.POINTER(ctypes.c_uint8)),
                ("node", ctypes.POINTER(_i32)), ("material", ctypes.POINTER(ctypes.c_uint8))]


class Nf2ffDesc(ctypes.Structure):
    _fields_ = [("n_freq", _i32), ("batch", _i32), ("task_s", (_i32 * 3) * 6),
                ("task_e", (_i32 * 3) * 6), ("te", _dp), ("th", _dp), ("scale", ctypes.c_double)]


class Nf2ffStepDesc(ctypes.Structure):
    """xfd_nf2ff_step_desc: one allocation-free NF2FF step on caller arrays."""
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("precision", _i32),
                ("fields", ctypes.c_void_p * 6), ("n_freq", _i32),
                ("task_s", (_i32 * 3) * 6), ("task_e", (_i32 * 3) * 6),
                ("te", ctypes.c_void_p), ("th", ctypes.c_void_p), ("n_steps", _i64),
                ("step", _i64), ("scale", ctypes.c_double), ("acc", ctypes.c_void_p),
                ("acc_comp", ctypes.c_void_p)]


class FarFieldDesc(ctypes.Structure):
    """xfd_far_field_desc."""
    _fields_ = [("n_angles", _i32), ("theta", _dp), ("phi", _dp), ("n_freq", _i32),
                ("freqs", _dp), ("origin", ctypes.c_double * 3), ("node_e", _dp * 3),
                ("node_h", _dp * 3), ("size_e", _dp * 3)]


class EngineError(RuntimeError):
    pass


_LIB = None


def library_path() -> str:
    return _build.ENGINE_LIB


def load(build_if_missing: bool = True):
    """Loads libxfd_engine.so (building it first if absent and nvcc exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.ENGINE_LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise EngineError(f"engine library not built: {path}")
        _build.build_engine()
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "xfd_create": ([ctypes.POINTER(GridDesc), ctypes.POINTER(vp)], ctypes.c_int),
        "xfd_destroy": ([vp], None),
        "xfd_last_error": ([vp], ctypes.c_char_p),
        "xfd_set_material_classes": ([vp, _dp, _i32, ctypes.POINTER(ctypes.c_uint16)],
                                     ctypes.c_int),
        "xfd_set_curl_factors": ([vp, _dp * 3, _dp * 3], ctypes.c_int),
        "xfd_add_cpml": ([vp, ctypes.POINTER(CpmlSlab)], ctypes.c_int),
        "xfd_set_tfsf": ([vp, ctypes.POINTER(TfsfDesc)], ctypes.c_int),
        "xfd_set_tfsf_slab": ([vp, ctypes.POINTER(TfsfDesc), _i32], ctypes.c_int),
        "xfd_add_current_source": ([vp, _i32, _i32 * 3, _i32 * 3, _dp, _dp], ctypes.c_int),
        "xfd_add_inductor": ([vp, _i32, _i32 * 3, _i32 * 3, _dp, _dp], ctypes.c_int),
        "xfd_set_ade": ([vp, ctypes.POINTER(AdeDesc)], ctypes.c_int),
        "xfd_set_nf2ff": ([vp, ctypes.POINTER(Nf2ffDesc)], ctypes.c_int),
        "xfd_get_nf2ff": ([vp, _dp, _i64, ctypes.POINTER(_i64)], ctypes.c_int),
        "xfd_add_movie": ([vp, _i32, _i32 * 3, _i32 * 3, _i32, ctypes.POINTER(_i32)],
                          ctypes.c_int),
        "xfd_get_movie_frames": ([vp, _i32, vp, _i64, ctypes.POINTER(_i64)], ctypes.c_int),
        "xfd_upload_fields": ([vp, vp * 6], ctypes.c_int),
        "xfd_download_fields": ([vp, vp * 6], ctypes.c_int),
        "xfd_download_field": ([vp, _i32, vp], ctypes.c_int),
        "xfd_run": ([vp, _i64], ctypes.c_int),
        "xfd_sync": ([vp], ctypes.c_int),
        "xfd_current_step": ([vp], _i64),
        "xfd_set_option": ([vp, ctypes.c_char_p, _i64], ctypes.c_int),
        "xfd_get_option": ([vp, ctypes.c_char_p, ctypes.POINTER(_i64)], ctypes.c_int),
        "xfd_nf2ff_step_static": ([ctypes.POINTER(Nf2ffStepDesc), vp], ctypes.c_int),
        "xfd_nf2ff_far_field": ([vp, ctypes.POINTER(FarFieldDesc), _dp, _i64], ctypes.c_int),
        "xfd_stream": ([vp], vp),
        "xfd_launches_per_step": ([vp], _i32),
        "xfd_stencil_bytes_per_step": ([vp], _i64),
        "xfd_algorithmic_bytes_per_step": ([vp], _i64),
        "xfd_set_e_overrides": ([vp, _i64, ctypes.POINTER(_i32), ctypes.POINTER(_i32), _dp, _dp],
                                ctypes.c_int),
        "xfd_set_h_term_overrides": ([vp, _i64, ctypes.POINTER(_i32), ctypes.POINTER(_i32), _dp,
                                      _dp], ctypes.c_int),
        "xfd_halo_copy": ([vp, _i32, vp, _i32, _i32, ctypes.POINTER(_i32)], ctypes.c_int),
        "xfd_plane_copy": ([vp, _i32, _i32, ctypes.POINTER(_i32), vp, _i32], ctypes.c_int),
        "xfd_plane_values": ([vp], _i64),
        "xfd_checkpoint_save": ([vp, _i32], ctypes.c_int),
        "xfd_checkpoint_load": ([vp, _i32], ctypes.c_int),
        "xfd_checkpoint_drop": ([vp, _i32], ctypes.c_int),
        "xfd_checkpoint_step": ([vp, _i32], _i64),
        "xfd_adjoint_run": ([vp, vp, _dp, _dp], ctypes.c_int),
        "xfd_batch_create": ([ctypes.POINTER(vp), _i32, ctypes.POINTER(vp)], ctypes.c_int),
        "xfd_batch_destroy": ([vp], None),
        "xfd_batch_last_error": ([vp], ctypes.c_char_p),
        "xfd_batch_run": ([vp, _i64], ctypes.c_int),
        "xfd_batch_sync": ([vp], ctypes.c_int),
        "xfd_batch_set_option": ([vp, ctypes.c_char_p, _i64], ctypes.c_int),
        "xfd_batch_get_option": ([vp, ctypes.c_char_p, ctypes.POINTER(_i64)], ctypes.c_int),
        "xfd_batch_tuning": ([vp, ctypes.POINTER(_i32), _dp, _i32, ctypes.POINTER(_i32)],
                             ctypes.c_int),
        "xfd_batch_tuning_shapes": ([vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                     ctypes.POINTER(_i32), _dp, _i32, ctypes.POINTER(_i32)],
                                    ctypes.c_int),
        "xfd_batch_size": ([vp], _i32),
        "xfd_batch_launches_per_step": ([vp], _i32),
        "xfd_batch_stream": ([vp], vp),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def exported_symbols() -> List[str]:
    """Names declared in include/xfd_engine.h that the library must export."""
    return ["xfd_create", "xfd_destroy", "xfd_last_error", "xfd_set_material_classes",
            "xfd_set_curl_factors", "xfd_add_cpml", "xfd_set_tfsf", "xfd_set_tfsf_slab",
            "xfd_add_current_source",
            "xfd_add_inductor",
            "xfd_set_ade", "xfd_set_nf2ff", "xfd_get_nf2ff", "xfd_add_movie",
            "xfd_get_movie_frames", "xfd_upload_fields", "xfd_download_fields",
            "xfd_download_field", "xfd_run", "xfd_sync", "xfd_current_step", "xfd_set_option",
            "xfd_get_option", "xfd_nf2ff_step_static", "xfd_nf2ff_far_field", "xfd_stream",
            "xfd_launches_per_step", "xfd_stencil_bytes_per_step",
            "xfd_algorithmic_bytes_per_step", "xfd_set_e_overrides", "xfd_set_h_term_overrides", "xfd_halo_copy",
            "xfd_plane_copy", "xfd_plane_values",
            "xfd_checkpoint_save", "xfd_checkpoint_load", "xfd_checkpoint_drop",
            "xfd_checkpoint_step", "xfd_adjoint_run", "xfd_set_nf2ff_td", "xfd_get_nf2ff_td",
            "xfd_add_probe", "xfd_get_probe",
            "xfd_batch_create",
            "xfd_batch_destroy", "xfd_batch_last_error", "xfd_batch_run", "xfd_batch_sync",
            "xfd_batch_set_option", "xfd_batch_get_option", "xfd_batch_tuning",
            "xfd_batch_tuning_shapes",
            "xfd_batch_size", "xfd_batch_launches_per_step", "xfd_batch_stream"]


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def comp_shape(n: Sequence[int], c: int):
    """Reference shape of component c (0..5) on an (nx, ny, nz) grid."""
    ax = c % 3
    if c < 3:
        return tuple(n[d] if d == ax else n[d] + 1 for d in range(3))
    return tuple(n[d] + 1 if d == ax else n[d] for d in range(3))


class Engine:
    """Owning handle of one xfd_engine."""

    def __init__(self, nx: int, ny: int, nz: int, precision: int = FP64, n_steps: int = 1,
                 dt: float = 0.0, device: int = 0):
        self.L = load()
        self.n = (nx, ny, nz)
        self.precision = precision
        self.dtype = np.float64 if precision == FP64 else np.float32
        self.n_steps = n_steps
        g = GridDesc(nx, ny, nz, precision, n_steps, dt, device)
        h = ctypes.c_void_p()
        st = self.L.xfd_create(ctypes.byref(g), ctypes.byref(h))
        if st != 0:
            raise EngineError(f"xfd_create: {_STATUS.get(st, st)}: "
                              f"{self.L.xfd_last_error(None).decode()}")
        self.h = h
        self._keep: list = []

    # ------------------------------------------------------------ plumbing
    def _check(self, st: int, what: str):
        if st != 0:
            msg = self.L.xfd_last_error(self.h).decode()
            raise EngineError(f"{what}: {_STATUS.get(st, st)}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.xfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------------- set-up
    def set_material_classes(self, table: np.ndarray, lattice_class: np.ndarray):
        table = _f64(table).reshape(-1, 12)
        lc = np.ascontiguousarray(lattice_class, dtype=np.uint16)
        assert lc.shape == (self.n[0] + 1, self.n[1] + 1, self.n[2] + 1), lc.shape
        self._check(self.L.xfd_set_material_classes(
            self.h, _p(table), table.shape[0],
            lc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))), "set_material_classes")

    def set_curl_factors(self, fe: Sequence[np.ndarray], fh: Sequence[np.ndarray]):
        fe = [_f64(a) for a in fe]
        fh = [_f64(a) for a in fh]
        ae = (_dp * 3)(*[_p(a) for a in fe])
        ah = (_dp * 3)(*[_p(a) for a in fh])
        self._check(self.L.xfd_set_curl_factors(self.h, ae, ah), "set_curl_factors")

    def add_cpml(self, axis: int, negative: bool, thickness: int, e_start: int, h_start: int,
                 a_e, b_e, a_h, b_h):
        arrs = [_f64(a) for a in (a_e, b_e, a_h, b_h)]
        s = CpmlSlab(axis, int(negative), thickness, e_start, h_start, *[_p(a) for a in arrs])
        self._check(self.L.xfd_add_cpml(self.h, ctypes.byref(s)), "add_cpml")

    def set_tfsf(self, box_s, box_e, e_inc, h_inc, p_int, p_half, ca, cb, te, th,
                 x_offset=None):
        """TFSF3D (xfd_set_tfsf); with x_offset, the source of a global lattice
        on the x-slab whose plane 0 is global plane x_offset (xfd_set_tfsf_slab)."""
        e_inc, h_inc = _f64(e_inc), _f64(h_inc)
        p_int = [_f64(a) for a in p_int]
        p_half = [_f64(a) for a in p_half]
        d = TfsfDesc()
        for a in range(3):
            d.box_s[a], d.box_e[a] = int(box_s[a]), int(box_e[a])
            d.p_int[a], d.p_half[a] = _p(p_int[a]), _p(p_half[a])
            d.ca[a], d.cb[a], d.te[a], d.th[a] = ca[a], cb[a], te[a], th[a]
        d.aux = e_inc.shape[1]
        d.e_inc, d.h_inc = _p(e_inc), _p(h_inc)
        if x_offset is None:
            self._check(self.L.xfd_set_tfsf(self.h, ctypes.byref(d)), "set_tfsf")
        else:
            self._check(self.L.xfd_set_tfsf_slab(self.h, ctypes.byref(d), int(x_offset)),
                        "set_tfsf_slab")

    def add_current_source(self, comp: int, box_s, box_e, coff, waveform):
        coff, waveform = _f64(coff), _f64(waveform)
        self._check(self.L.xfd_add_current_source(
            self.h, comp, (_i32 * 3)(*box_s), (_i32 * 3)(*box_e), _p(coff), _p(waveform)),
            "add_current_source")

    def add_inductor(self, comp: int, box_s, box_e, cecjc, cjcec):
        cecjc, cjcec = _f64(cecjc), _f64(cjcec)
        self._check(self.L.xfd_add_inductor(
            self.h, comp, (_i32 * 3)(*box_s), (_i32 * 3)(*box_e), _p(cecjc), _p(cjcec)),
            "add_inductor")

    def set_ade(self, kind: int, n_poles: int, mat_coeff: np.ndarray, comp: np.ndarray,
                node: np.ndarray, material: np.ndarray):
        mc = _f64(mat_coeff).ravel()
        comp = np.ascontiguousarray(comp, dtype=np.uint8)
        node = np.ascontiguousarray(node, dtype=np.int32).reshape(-1, 3)
        material = np.ascontiguousarray(material, dtype=np.uint8)
        n_mat = mc.size // (2 + 7 * n_poles)
        d = AdeDesc(kind, n_poles, n_mat, _p(mc), comp.size,
                    comp.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                    node.ctypes.data_as(ctypes.POINTER(_i32)),
                    material.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        self._check(self.L.xfd_set_ade(self.h, ctypes.byref(d)), "set_ade")

    def set_nf2ff(self, tasks, te: np.ndarray, th: np.ndarray, scale: float, batch: int = 64):
        te, th = _f64(te), _f64(th)
        d = Nf2ffDesc()
        d.n_freq = te.shape[0]
        d.batch = batch
        for f in range(6):
            t = tasks[f]
            for a in range(3):
                d.task_s[f][a] = 0 if t is None else int(t[0][a])
                d.task_e[f][a] = 0 if t is None else int(t[1][a])
        d.te, d.th, d.scale = _p(te), _p(th), float(scale)
        self._check(self.L.xfd_set_nf2ff(self.h, ctypes.byref(d)), "set_nf2ff")

    def add_movie(self, field: int, box_s, box_e, interval: int) -> int:
        out = _i32()
        self._check(self.L.xfd_add_movie(self.h, field, (_i32 * 3)(*box_s), (_i32 * 3)(*box_e),
                                         interval, ctypes.byref(out)), "add_movie")
        return out.value

    def set_option(self, name: str, value: int):
        self._check(self.L.xfd_set_option(self.h, name.encode(), int(value)), "set_option")

    def get_option(self, name: str) -> int:
        v = _i64()
        self._check(self.L.xfd_get_option(self.h, name.encode(), ctypes.byref(v)), "get_option")
        return int(v.value)

    # ---------------------------------------------------------------- fields
    def upload_fields(self, fields: Sequence[np.ndarray]):
        arrs = []
        for c in range(6):
            a = np.ascontiguousarray(fields[c], dtype=self.dtype)
            assert a.shape == comp_shape(self.n, c), (c, a.shape)
            arrs.append(a)
        ptrs = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in arrs])
        self._check(self.L.xfd_upload_fields(self.h, ptrs), "upload_fields")

    def download_fields(self) -> List[np.ndarray]:
        arrs = [np.empty(comp_shape(self.n, c), dtype=self.dtype) for c in range(6)]
        ptrs = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in arrs])
        self._check(self.L.xfd_download_fields(self.h, ptrs), "download_fields")
        return arrs

    def download_field(self, c: int) -> np.ndarray:
        a = np.empty(comp_shape(self.n, c), dtype=self.dtype)
        self._check(self.L.xfd_download_field(self.h, c, ctypes.c_void_p(a.ctypes.data)),
                    "download_field")
        return a

    # ------------------------------------------------------------------- run
    def run(self, n: int):
        self._check(self.L.xfd_run(self.h, int(n)), "run")

    def sync(self):
        self._check(self.L.xfd_sync(self.h), "sync")

    @property
    def step(self) -> int:
        return int(self.L.xfd_current_step(self.h))

    def halo_copy_from(self, dst_plane: int, src: "Engine", src_plane: int,
                       comps: Sequence[int]):
        """xfd_halo_copy: planes of `src`'s current fields into this engine's."""
        arr = (_i32 * len(comps))(*comps)
        self._check(self.L.xfd_halo_copy(self.h, int(dst_plane), src.h, int(src_plane),
                                         len(comps), arr), "halo_copy")

    def plane_values(self) -> int:
        """xfd_plane_values: values of one padded x-plane (NY x KP)."""
        return int(self.L.xfd_plane_values(self.h))

    def plane_copy(self, plane: int, comps: Sequence[int], buf_ptr: int, into_engine: bool):
        """xfd_plane_copy: x-plane `plane` of components `comps` between this
        engine's current fields and the buffer at `buf_ptr` (device or host,
        len(comps) x plane_values() values of the engine's precision)."""
        arr = (_i32 * len(comps))(*comps)
        self._check(self.L.xfd_plane_copy(self.h, int(plane), len(comps), arr,
                                          ctypes.c_void_p(int(buf_ptr)), 1 if into_engine else 0),
                    "plane_copy")

    def stream(self) -> int:
        return int(self.L.xfd_stream(self.h) or 0)

    def launches_per_step(self) -> int:
        return int(self.L.xfd_launches_per_step(self.h))

    def stencil_bytes_per_step(self) -> int:
        return int(self.L.xfd_stencil_bytes_per_step(self.h))

    # ------------------------------------------------------- saved states
    def checkpoint_save(self, slot: int):
        self._check(self.L.xfd_checkpoint_save(self.h, int(slot)), "checkpoint_save")

    def checkpoint_load(self, slot: int):
        self._check(self.L.xfd_checkpoint_load(self.h, int(slot)), "checkpoint_load")

    def checkpoint_drop(self, slot: int):
        self._check(self.L.xfd_checkpoint_drop(self.h, int(slot)), "checkpoint_drop")

    def checkpoint_step(self, slot: int) -> int:
        return int(self.L.xfd_checkpoint_step(self.h, int(slot)))

    # --------------------------------------------------------------- outputs
    def movie_frames(self, mid: int, box_shape) -> np.ndarray:
        n = _i64()
        self._check(self.L.xfd_get_movie_frames(self.h, mid, None, 0, ctypes.byref(n)),
                    "get_movie_frames")
        out = np.empty((n.value, *box_shape), dtype=self.dtype)
        self._check(self.L.xfd_get_movie_frames(self.h, mid, ctypes.c_void_p(out.ctypes.data),
                                                out.nbytes, ctypes.byref(n)),
                    "get_movie_frames")
        return out

    def nf2ff(self) -> np.ndarray:
        cnt = _i64()
        self._check(self.L.xfd_get_nf2ff(self.h, None, 0, ctypes.byref(cnt)), "get_nf2ff")
        out = np.empty(2 * cnt.value, dtype=np.float64)
        self._check(self.L.xfd_get_nf2ff(self.h, _p(out), cnt.value, ctypes.byref(cnt)),
                    "get_nf2ff")
        return out[0::2] + 1j * out[1::2]


def nf2ff_step_static(n, precision: int, fields, tasks, te_dev: int, th_dev: int, n_freq: int,
                      n_steps: int, step: int, scale: float, acc_dev: int, stream: int = 0,
                      acc_comp_dev: int = 0):
    """Folds one time step of the Huygens-surface fields into `acc_dev` through
    xfd_nf2ff_step_static, the entry point that allocates no device memory
    (for callers whose device memory belongs to another allocator).  `fields`
    are six device addresses of the component arrays in the reference shapes;
    te_dev/th_dev/acc_dev are device addresses of complex128 arrays;
    `acc_comp_dev` (optional, shaped like acc, zeroed before the first step)
    turns on compensated accumulation (the sum is acc + acc_comp)."""
    L = load()
    d = Nf2ffStepDesc()
    d.nx, d.ny, d.nz = (int(x) for x in n)
    d.precision = int(precision)
    for c in range(6):
        d.fields[c] = int(fields[c])
    d.n_freq = int(n_freq)
    for f in range(6):
        t = tasks[f]
        for a in range(3):
            d.task_s[f][a] = 0 if t is None else int(t[0][a])
            d.task_e[f][a] = 0 if t is None else int(t[1][a])
    d.te, d.th, d.acc = int(te_dev), int(th_dev), int(acc_dev)
    d.acc_comp = int(acc_comp_dev) if acc_comp_dev else None
    d.n_steps, d.step, d.scale = int(n_steps), int(step), float(scale)
    st = L.xfd_nf2ff_step_static(ctypes.byref(d), ctypes.c_void_p(int(stream)))
    if st != 0:
        raise EngineError(f"xfd_nf2ff_step_static: {L.xfd_last_error(None).decode()} (status {st})")


class Batch:
    """Owning handle of one xfd_batch over borrowed engine handles.

    ``engines`` are raw xfd_engine pointers (``Engine.h`` or
    ``SceneRun.engine_handle()``); their owners must outlive the batch.
    """

    def __init__(self, engines: Sequence[int], options: Optional[Dict[str, int]] = None):
        self.L = load()
        arr = (ctypes.c_void_p * len(engines))(*[int(e) for e in engines])
        h = ctypes.c_void_p()
        st = self.L.xfd_batch_create(arr, len(engines), ctypes.byref(h))
        if st != 0:
            raise EngineError(f"xfd_batch_create: {_STATUS.get(st, st)}: "
                              f"{self.L.xfd_batch_last_error(None).decode()}")
        self.h = h
        for name, value in (options or {}).items():
            self.set_option(name, value)

    def _check(self, st: int, what: str):
        if st != 0:
            msg = self.L.xfd_batch_last_error(self.h).decode()
            raise EngineError(f"{what}: {_STATUS.get(st, st)}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.xfd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n: int):
        self._check(self.L.xfd_batch_run(self.h, int(n)), "batch_run")

    def sync(self):
        self._check(self.L.xfd_batch_sync(self.h), "batch_sync")

    def set_option(self, name: str, value: int):
        self._check(self.L.xfd_batch_set_option(self.h, name.encode(), int(value)),
                    "batch_set_option")

    def get_option(self, name: str) -> int:
        v = _i64()
        self._check(self.L.xfd_batch_get_option(self.h, name.encode(), ctypes.byref(v)),
                    "batch_get_option")
        return int(v.value)

    def tuning(self) -> List[tuple]:
        """(tile depth, ms per batch step) of the last autotuning."""
        cnt = _i32()
        self._check(self.L.xfd_batch_tuning(self.h, None, None, 0, ctypes.byref(cnt)),
                    "batch_tuning")
        d = (_i32 * max(cnt.value, 1))()
        ms = np.zeros(max(cnt.value, 1))
        self._check(self.L.xfd_batch_tuning(self.h, d, _p(ms), cnt.value, ctypes.byref(cnt)),
                    "batch_tuning")
        return [(int(d[q]), float(ms[q])) for q in range(cnt.value)]

    def tuning_shapes(self) -> List[tuple]:
        """(queue form, tile rows, tile depth, ms per batch step) of the last
        autotuning."""
        cnt = _i32()
        self._check(self.L.xfd_batch_tuning_shapes(self.h, None, None, None, None, 0,
                                                   ctypes.byref(cnt)), "batch_tuning_shapes")
        n = max(cnt.value, 1)
        qf, r, d = (_i32 * n)(), (_i32 * n)(), (_i32 * n)()
        ms = np.zeros(n)
        self._check(self.L.xfd_batch_tuning_shapes(self.h, qf, r, d, _p(ms), cnt.value,
                                                   ctypes.byref(cnt)), "batch_tuning_shapes")
        return [(int(qf[q]), int(r[q]), int(d[q]), float(ms[q])) for q in range(cnt.value)]

    def size(self) -> int:
        return int(self.L.xfd_batch_size(self.h))

    def launches_per_step(self) -> int:
        return int(self.L.xfd_batch_launches_per_step(self.h))

    def stream(self) -> int:
        return int(self.L.xfd_batch_stream(self.h) or 0)
