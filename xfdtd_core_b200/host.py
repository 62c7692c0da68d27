"""ctypes binding of the host library's C entry points (include/xfdtd_host.h).

A :class:`SceneRun` is one ``xfdtd::Simulation`` built from a
:class:`xfdtd_core_b200.scene.Scene` by the C++20 host library, which does the
FP64 set-up and drives the CUDA engine.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from typing import List, Optional, Tuple

import numpy as np

from . import build as _build
from . import engine as _engine

NO_ENGINE = 0x100
_dp = ctypes.POINTER(ctypes.c_double)
_LIB = None


class HostError(RuntimeError):
    pass


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(_build.HOST_LIB):
        _build.build_engine()
        _build.build_host()
    L = ctypes.CDLL(_build.HOST_LIB)
    vp = ctypes.c_void_p
    i32, i64 = ctypes.c_int32, ctypes.c_int64
    sig = {
        "xfdtd_scene_open": ([ctypes.c_char_p, i32, ctypes.POINTER(vp)], ctypes.c_int),
        "xfdtd_scene_close": ([vp], None),
        "xfdtd_host_last_error": ([], ctypes.c_char_p),
        "xfdtd_scene_engine": ([vp], vp),
        "xfdtd_scene_set_engine_option": ([vp, ctypes.c_char_p, i64], ctypes.c_int),
        "xfdtd_scene_info": ([vp, i32 * 3, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(i64)], ctypes.c_int),
        "xfdtd_scene_advance": ([vp, i64], ctypes.c_int),
        "xfdtd_scene_finish": ([vp], ctypes.c_int),
        "xfdtd_scene_coefficients": ([vp, _dp * 18], ctypes.c_int),
        "xfdtd_scene_field": ([vp, i32, _dp], ctypes.c_int),
        "xfdtd_scene_tfsf": ([vp, _dp, _dp, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.POINTER(i32)], ctypes.c_int),
        "xfdtd_scene_movie": ([vp, i32, _dp, i64, ctypes.POINTER(i64), i32 * 3], ctypes.c_int),
        "xfdtd_scene_nf2ff": ([vp, _dp, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "xfdtd_scene_far_field": ([vp, i32, _dp, i32, _dp, _dp, _dp, i64, ctypes.POINTER(i64),
                                   ctypes.c_char_p, ctypes.c_char_p], ctypes.c_int),
        "xfdtd_scene_field_time": ([vp, i32, _dp, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "xfdtd_scene_write_outputs": ([vp, ctypes.c_char_p], ctypes.c_int),
        "xfdtd_scene_dft_objective": ([vp, i64, i32, i32 * 3, i32 * 3, ctypes.c_double, i32, i32,
                                       _dp, _dp, i64], ctypes.c_int),
        "xfdtd_scene_nf2ff_td": ([vp, _dp, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "xfdtd_scene_line_monitor": ([vp, i32, i32, _dp, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "xfdtd_scene_s_parameter": ([vp, i32, _dp, i64, ctypes.POINTER(i64)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def exported_symbols() -> List[str]:
    return ["xfdtd_scene_open", "xfdtd_scene_close", "xfdtd_host_last_error",
            "xfdtd_scene_engine", "xfdtd_scene_set_engine_option", "xfdtd_scene_info",
            "xfdtd_scene_advance", "xfdtd_scene_tfsf", "xfdtd_scene_finish",
            "xfdtd_scene_coefficients", "xfdtd_scene_field", "xfdtd_scene_movie",
            "xfdtd_scene_nf2ff", "xfdtd_scene_far_field", "xfdtd_scene_field_time",
            "xfdtd_scene_write_outputs", "xfdtd_scene_dft_objective", "xfdtd_scene_nf2ff_td",
            "xfdtd_scene_line_monitor", "xfdtd_scene_s_parameter"]


class SceneRun:
    """A Simulation built from a scene by the C++ host library."""

    def __init__(self, scene, precision: int = 0, engine: bool = True,
                 options: Optional[dict] = None):
        self.L = load()
        self.scene = scene
        fd, self.path = tempfile.mkstemp(suffix=".scene")
        with os.fdopen(fd, "w") as fh:
            fh.write(scene.to_text())
        h = ctypes.c_void_p()
        flags = precision | (0 if engine else NO_ENGINE)
        st = self.L.xfdtd_scene_open(self.path.encode(), flags, ctypes.byref(h))
        os.unlink(self.path)
        if st != 0:
            raise HostError(self.L.xfdtd_host_last_error().decode())
        self.h = h
        n = (ctypes.c_int32 * 3)()
        dt = ctypes.c_double()
        steps = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_info(self.h, n, ctypes.byref(dt), ctypes.byref(steps)))
        self.n = tuple(n)
        self.dt = dt.value
        self.steps = steps.value
        for name, value in (options or {}).items():
            self.set_engine_option(name, value)

    def set_engine_option(self, name: str, value: int):
        """Engine option (graph, graph_chunk, kernel, ichunk)."""
        self._check(self.L.xfdtd_scene_set_engine_option(self.h, name.encode(), int(value)))

    def get_engine_option(self, name: str) -> int:
        """The engine's current value of an option (xfd_get_option)."""
        import ctypes
        from xfdtd_core_b200 import engine as E
        v = ctypes.c_int64()
        L = E.load()
        if L.xfd_get_option(ctypes.c_void_p(self.engine_handle()), name.encode(),
                            ctypes.byref(v)) != 0:
            raise HostError(L.xfd_last_error(ctypes.c_void_p(self.engine_handle())).decode())
        return int(v.value)

    def _check(self, st):
        if st != 0:
            raise HostError(self.L.xfdtd_host_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.xfdtd_scene_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def engine_handle(self) -> int:
        return int(self.L.xfdtd_scene_engine(self.h) or 0)

    def advance(self, n: int):
        self._check(self.L.xfdtd_scene_advance(self.h, int(n)))

    def finish(self):
        self._check(self.L.xfdtd_scene_finish(self.h))

    def run(self, n: Optional[int] = None):
        self.advance(self.steps if n is None else n)
        self.finish()

    def coefficients(self) -> List[np.ndarray]:
        """cexe cexhy cexhz ceye ceyhz ceyhx ceze cezhx cezhy chxh chxey chxez
        chyh chyez chyex chzh chzex chzey, reference shapes."""
        shapes = []
        for c in range(6):
            s = _engine.comp_shape(self.n, c)
            shapes += [s, s, s]
        arrs = [np.empty(s) for s in shapes]
        ptrs = (_dp * 18)(*[a.ctypes.data_as(_dp) for a in arrs])
        self._check(self.L.xfdtd_scene_coefficients(self.h, ptrs))
        return arrs

    def tfsf_tables(self, box_size):
        """(e_inc, h_inc, p_int[3], p_half[3]) the host computed, or None."""
        aux = ctypes.c_int32()
        self._check(self.L.xfdtd_scene_tfsf(self.h, None, None, None, None, ctypes.byref(aux)))
        if aux.value == 0:
            return None
        e_inc = np.empty((self.steps, aux.value))
        h_inc = np.empty((self.steps, aux.value - 1))
        p_int = [np.empty(box_size[a] + 1) for a in range(3)]
        p_half = [np.empty(box_size[a] + 2) for a in range(3)]
        pi = (_dp * 3)(*[x.ctypes.data_as(_dp) for x in p_int])
        ph = (_dp * 3)(*[x.ctypes.data_as(_dp) for x in p_half])
        self._check(self.L.xfdtd_scene_tfsf(self.h, e_inc.ctypes.data_as(_dp),
                                            h_inc.ctypes.data_as(_dp), ctypes.cast(pi, ctypes.c_void_p),
                                            ctypes.cast(ph, ctypes.c_void_p), ctypes.byref(aux)))
        return e_inc, h_inc, p_int, p_half

    def field(self, c: int) -> np.ndarray:
        a = np.empty(_engine.comp_shape(self.n, c))
        self._check(self.L.xfdtd_scene_field(self.h, c, a.ctypes.data_as(_dp)))
        return a

    def fields(self) -> List[np.ndarray]:
        return [self.field(c) for c in range(6)]

    def movie(self, index: int = 0) -> np.ndarray:
        nfr = ctypes.c_int64()
        shp = (ctypes.c_int32 * 3)()
        self._check(self.L.xfdtd_scene_movie(self.h, index, None, 0, ctypes.byref(nfr), shp))
        out = np.empty((nfr.value, *tuple(shp)))
        self._check(self.L.xfdtd_scene_movie(self.h, index, out.ctypes.data_as(_dp), out.size,
                                             ctypes.byref(nfr), shp))
        return out

    def field_time(self, index: int = 0) -> np.ndarray:
        """[time; samples] of field time monitor `index`, shape (2, steps)."""
        cnt = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_field_time(self.h, index, None, 0, ctypes.byref(cnt)))
        out = np.empty(2 * cnt.value)
        self._check(self.L.xfdtd_scene_field_time(self.h, index, out.ctypes.data_as(_dp),
                                                  out.size, ctypes.byref(cnt)))
        return out.reshape(2, cnt.value)

    def nf2ff(self) -> np.ndarray:
        cnt = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_nf2ff(self.h, None, 0, ctypes.byref(cnt)))
        out = np.empty(2 * cnt.value)
        self._check(self.L.xfdtd_scene_nf2ff(self.h, out.ctypes.data_as(_dp), cnt.value,
                                             ctypes.byref(cnt)))
        return out[0::2] + 1j * out[1::2]

    def far_field(self, theta, phi, origin=(0.0, 0.0, 0.0), directory: Optional[str] = None,
                  sub_dir: Optional[str] = None) -> np.ndarray:
        """Far-field potentials computed on the GPU: complex
        [n_freq, 4 (a_theta, f_phi, a_phi, f_theta), n_angles]; with `sub_dir`
        the per-frequency .npy files of processFarField are written too."""
        th = np.ascontiguousarray(np.atleast_1d(theta), dtype=np.float64)
        ph = np.ascontiguousarray(np.atleast_1d(phi), dtype=np.float64)
        org = np.ascontiguousarray(origin, dtype=np.float64)
        cnt = ctypes.c_int64()
        args = (self.h, th.size, th.ctypes.data_as(_dp), ph.size, ph.ctypes.data_as(_dp),
                org.ctypes.data_as(_dp))
        self._check(self.L.xfdtd_scene_far_field(*args, None, 0, ctypes.byref(cnt), None, None))
        out = np.empty(2 * cnt.value)
        self._check(self.L.xfdtd_scene_far_field(
            *args, out.ctypes.data_as(_dp), cnt.value, ctypes.byref(cnt),
            directory.encode() if directory else None, sub_dir.encode() if sub_dir else None))
        n_ang = th.size * ph.size
        return (out[0::2] + 1j * out[1::2]).reshape(-1, 4, n_ang)

    def dft_objective(self, n_steps: int, field: int, box_s, box_e, freq: float,
                      grad: bool = False, voxel_object: int = 0,
                      checkpoint_interval: int = 250):
        """J = sum_p |F_p|^2, F_p = dt sum_n E^n(p) exp(-i 2 pi freq n dt) over the
        next n_steps steps at the nodes of [box_s, box_e) of E component
        `field`; with grad=True also dJ/deps_r per voxel of the VoxelObject
        (discrete adjoint).  Returns J, or (J, grad array in the voxel shape)."""
        J = ctypes.c_double()
        bs = (ctypes.c_int32 * 3)(*box_s)
        be = (ctypes.c_int32 * 3)(*box_e)
        if not grad:
            self._check(self.L.xfdtd_scene_dft_objective(self.h, int(n_steps), field, bs, be,
                                                         float(freq), voxel_object,
                                                         checkpoint_interval, ctypes.byref(J),
                                                         None, 0))
            return J.value
        vox = [o for o in self.scene.objects if hasattr(o, "voxel_index")][voxel_object]
        g = np.zeros(np.asarray(vox.eps_r).shape)
        self._check(self.L.xfdtd_scene_dft_objective(
            self.h, int(n_steps), field, bs, be, float(freq), voxel_object, checkpoint_interval,
            ctypes.byref(J), g.ctypes.data_as(_dp), g.size))
        return J.value, g

    def line_monitor(self, kind: str, index: int = 0) -> np.ndarray:
        """[time; data] (2 x n_steps) of voltage (kind "voltage") or current
        monitor number `index`."""
        k = {"voltage": 0, "current": 1}[kind]
        cnt = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_line_monitor(self.h, k, index, None, 0, ctypes.byref(cnt)))
        out = np.zeros(cnt.value)
        self._check(self.L.xfdtd_scene_line_monitor(self.h, k, index, out.ctypes.data_as(_dp),
                                                    cnt.value, ctypes.byref(cnt)))
        return out.reshape(2, -1)

    def s_parameter(self, key: int) -> np.ndarray:
        """S[key] (key = 10 j + i) of the scene's network, per frequency."""
        cnt = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_s_parameter(self.h, key, None, 0, ctypes.byref(cnt)))
        out = np.zeros(cnt.value)
        self._check(self.L.xfdtd_scene_s_parameter(self.h, key, out.ctypes.data_as(_dp),
                                                   cnt.value, ctypes.byref(cnt)))
        return out[0::2] + 1j * out[1::2]

    def nf2ff_td(self) -> dict:
        """Time-domain NF2FF far-field series (w_theta, w_phi, u_theta, u_phi)."""
        cnt = ctypes.c_int64()
        self._check(self.L.xfdtd_scene_nf2ff_td(self.h, None, 0, ctypes.byref(cnt)))
        out = np.zeros(cnt.value)
        self._check(self.L.xfdtd_scene_nf2ff_td(self.h, out.ctypes.data_as(_dp), cnt.value,
                                                ctypes.byref(cnt)))
        n = cnt.value // 4
        return {k: out[q * n:(q + 1) * n] for q, k in
                enumerate(("w_theta", "w_phi", "u_theta", "u_phi"))}

    def write_outputs(self, directory: str):
        self._check(self.L.xfdtd_scene_write_outputs(self.h, directory.encode()))
