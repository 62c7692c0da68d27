"""Seeded kernel-level cases: one random configuration expressed twice, as
engine inputs (material classes + curl factors + compact slabs/lists) and as
oracle inputs (the reference's 18 full-grid coefficient arrays, full-grid
CPML/ADE arrays), so that each CUDA kernel is checked against the oracle's
restatement of the reference loops on identical numbers."""
from __future__ import annotations

import numpy as np

from xfdtd_core_b200.engine import comp_shape


def tan_a(c):
    return (c + 1) % 3


def tan_b(c):
    return (c + 2) % 3


class KernelCase:
    def __init__(self, n=(9, 10, 11), n_classes=5, seed=0,
                 slabs=((0, True, 3), (0, False, 2), (1, True, 2), (1, False, 3), (2, True, 2),
                        (2, False, 2)),
                 field_scale=1.0):
        rng = np.random.default_rng(seed)
        self.rng = rng
        self.n = tuple(n)
        nx, ny, nz = self.n
        table = np.empty((n_classes, 12))
        table[:, 0::2] = rng.uniform(0.85, 1.0, (n_classes, 6))
        table[:, 1::2] = rng.uniform(0.15, 0.5, (n_classes, 6))
        self.table = table
        self.lattice_class = rng.integers(0, n_classes, (nx + 1, ny + 1, nz + 1)).astype(np.uint16)
        self.fe = [rng.uniform(0.5, 1.5, self.n[a] + 1) for a in range(3)]
        self.fh = [rng.uniform(0.5, 1.5, self.n[a]) for a in range(3)]
        self.fields = [rng.standard_normal(comp_shape(self.n, c)) * field_scale for c in range(6)]
        self.slabs = []
        for (m, neg, thick) in slabs:
            e_start = 1 if neg else self.n[m] - thick
            h_start = 0 if neg else self.n[m] - thick
            self.slabs.append({
                "m": m, "neg": neg, "n": thick, "e_start": e_start, "h_start": h_start,
                "a_e": rng.uniform(-0.3, -0.01, thick), "b_e": rng.uniform(0.5, 0.99, thick),
                "a_h": rng.uniform(-0.3, -0.01, thick), "b_h": rng.uniform(0.5, 0.99, thick)})
        self.tfsf = None
        self.lumped = []
        self.ade = None
        self.nf2ff = None

    @classmethod
    def from_setup(cls, setup):
        """A case over explicit engine inputs (xfdtd_core_b200.slab.LocalSetup:
        one slab of a decomposed lattice), for its oracle and engine."""
        self = cls.__new__(cls)
        self.rng = np.random.default_rng(0)
        self.n = tuple(setup.n)
        self.table = setup.table
        self.lattice_class = setup.lattice_class
        self.fe, self.fh = list(setup.fe), list(setup.fh)
        self.fields = [np.array(f) for f in setup.fields]
        self.slabs = [dict(s) for s in setup.slabs]
        self.lumped = [dict(l) for l in setup.lumped]
        self.tfsf = getattr(setup, "tfsf", None)
        self.ade = getattr(setup, "ade", None)
        self.nf2ff = None
        return self

    # ------------------------------------------------------------- oracle
    def _cls_coeff(self, comp6: int):
        shp = comp_shape(self.n, comp6)
        cls = self.lattice_class[:shp[0], :shp[1], :shp[2]]
        return self.table[cls, 2 * comp6], self.table[cls, 2 * comp6 + 1]

    @staticmethod
    def _axis(vec, axis, shape):
        s = [1, 1, 1]
        s[axis] = shape[axis]
        return vec[:shape[axis]].reshape(s)

    def oracle_coefficients(self):
        ce, ceh_a, ceh_b, ch, che_a, che_b = [], [], [], [], [], []
        for c in range(3):
            ta, tb = tan_a(c), tan_b(c)
            shp = comp_shape(self.n, c)
            ca, cb = self._cls_coeff(c)
            ce.append(ca)
            ceh_a.append(-cb * self._axis(self.fe[tb], tb, shp))
            ceh_b.append(cb * self._axis(self.fe[ta], ta, shp))
            shp = comp_shape(self.n, 3 + c)
            ca, cb = self._cls_coeff(3 + c)
            ch.append(ca)
            che_a.append(cb * self._axis(self.fh[tb], tb, shp))
            che_b.append(-cb * self._axis(self.fh[ta], ta, shp))
        return ce, ceh_a, ceh_b, ch, che_a, che_b

    def oracle_pml(self):
        out = []
        for s in self.slabs:
            m, thick = s["m"], s["n"]
            A, B = tan_a(m), tan_b(m)
            nloc = list(self.n)
            nloc[m] = thick
            c_psi, psi = [], []
            # E_A (-cb), E_B (+cb), H_A (+cb), H_B (-cb) over their slab shapes.
            for q, (comp6, sign, start) in enumerate(
                    [(A, -1.0, s["e_start"]), (B, 1.0, s["e_start"]),
                     (3 + A, 1.0, s["h_start"]), (3 + B, -1.0, s["h_start"])]):
                shp = list(nloc)
                if q in (0, 3):
                    shp[B] += 1
                else:
                    shp[A] += 1
                sl = [slice(0, shp[0]), slice(0, shp[1]), slice(0, shp[2])]
                sl[m] = slice(start, start + thick)
                cls = self.lattice_class[tuple(sl)]
                cp = sign * self.table[cls, 2 * comp6 + 1]
                c_psi.append(np.ascontiguousarray(cp))
                psi.append(np.zeros(shp))
            task_s = [0, 0, 0]
            task_e = list(self.n)
            task_s[m], task_e[m] = s["h_start"], s["h_start"] + thick
            out.append({"m": m, "n": thick, "e_start": s["e_start"], "h_start": s["h_start"],
                        "task_s": task_s, "task_e": task_e, "a_e": s["a_e"], "b_e": s["b_e"],
                        "a_h": s["a_h"], "b_h": s["b_h"], "c_psi": c_psi, "psi": psi})
        return out

    def oracle(self):
        from oracle.reference_model import RefSimulation
        ce, ceh_a, ceh_b, ch, che_a, che_b = self.oracle_coefficients()
        return RefSimulation.from_arrays(
            self.n, [f.copy() for f in self.fields[:3]], [f.copy() for f in self.fields[3:]],
            ce, ceh_a, ceh_b, ch, che_a, che_b, pml=self.oracle_pml(), tfsf=self.tfsf,
            lumped=self.lumped, ade=self.oracle_ade(), nf2ff=self.oracle_nf2ff())

    # -------------------------------------------------------------- engine
    def engine(self, precision=0, n_steps=8, kernel=1, ichunk=None):
        """The case as an engine; kernel=None keeps the engine's own choice of
        sweep for the lattice."""
        from xfdtd_core_b200.engine import Engine
        eng = Engine(*self.n, precision=precision, n_steps=n_steps, dt=1.0)
        if kernel is not None:
            eng.set_option("kernel", kernel)
        if ichunk is not None:
            eng.set_option("ichunk", ichunk)
            eng.set_option("march_ichunk", ichunk)
        eng.set_material_classes(self.table, self.lattice_class)
        eng.set_curl_factors(self.fe, self.fh)
        for s in self.slabs:
            eng.add_cpml(s["m"], s["neg"], s["n"], s["e_start"], s["h_start"], s["a_e"],
                         s["b_e"], s["a_h"], s["b_h"])
        if self.tfsf is not None:
            t = self.tfsf
            eng.set_tfsf(t["box_s"], t["box_e"], t["e_inc"], t["h_inc"], t["p_int"],
                         t["p_half"], t["ca"], t["cb"], t["te"], t["th"],
                         x_offset=t.get("x_offset"))
        for l in self.lumped:
            eng.add_current_source(l["comp"], l["s"], l["e"], l["coff"], l["wave"])
        if self.ade is not None:
            a = self.ade
            eng.set_ade(a["kind"], a["np"], a["mat_coeff"], a["comp"], a["node"], a["material"])
        if self.nf2ff is not None:
            nf = self.nf2ff
            eng.set_nf2ff(nf["tasks"], nf["te"], nf["th"], scale=nf["nf"], batch=nf["batch"])
        eng.upload_fields([f.astype(eng.dtype) for f in self.fields])
        return eng

    # ---------------------------------------------------------- extensions
    def add_lumped(self, comp=2, s=(3, 4, 4), e=(5, 6, 6), n_steps=8):
        rng = self.rng
        shp = tuple(e[a] - s[a] for a in range(3))
        self.lumped.append({"comp": comp, "s": list(s), "e": list(e),
                            "coff": rng.standard_normal(shp),
                            "wave": rng.standard_normal(n_steps)})

    def add_ade(self, kind=0, n_poles=2, n_mat=2, frac=0.3, margin=0):
        """Random dispersive nodes: a random set of cells (none within
        `margin` cells of a lattice face), their three E components within
        the E update ranges, random per-material coefficients."""
        rng = self.rng
        nx, ny, nz = self.n
        cells = rng.random((nx, ny, nz)) < frac
        if margin:
            inner = np.zeros_like(cells)
            inner[margin:nx - margin, margin:ny - margin, margin:nz - margin] = True
            cells &= inner
        mat_of_cell = rng.integers(0, n_mat, (nx, ny, nz))
        coef = rng.uniform(-0.2, 0.2, (n_mat, 2 + 7 * n_poles))
        comp, node, material = [], [], []
        for c in range(3):
            lo = [0, 0, 0]
            lo[tan_a(c)] = 1
            lo[tan_b(c)] = 1
            idx = np.argwhere(cells)
            for (i, j, k) in idx:
                if i >= lo[0] and j >= lo[1] and k >= lo[2]:
                    comp.append(c)
                    node.append((i, j, k))
                    material.append(mat_of_cell[i, j, k])
        self.ade = {"kind": kind, "np": n_poles, "mat_coeff": coef, "comp": np.array(comp),
                    "node": np.array(node), "material": np.array(material),
                    "cells": cells, "mat_of_cell": mat_of_cell}

    def oracle_ade(self):
        """Full-grid ADE arrays with the per-material coefficients at the
        dispersive cells and zeros elsewhere.  The same cell-level coefficient
        serves Ex, Ey and Ez of the cell, as in the reference storage."""
        if self.ade is None:
            return None
        a = self.ade
        nx, ny, nz = self.n
        P = a["np"]
        cells, moc, coef = a["cells"], a["mat_of_cell"], a["mat_coeff"]
        z4 = lambda: np.zeros((nx, ny, nz, P))
        z3 = lambda: np.zeros((nx, ny, nz))
        st = {"kind": a["kind"], "np": P, "cejsum": z3(), "cjj": z4(), "cje": z4(),
              "cjsumj": z4(), "j": [z4() for _ in range(3)]}
        names = ["cjj", "cjjp", "cjen", "cje", "cjep", "cjsumj", "cjsumjp"]
        if a["kind"] == 0:
            for nm in ("cjjp", "cjen", "cjep", "cjsumjp"):
                st[nm] = z4()
            st["ceep"] = z3()
            st["eprev"] = [z3() for _ in range(3)]
            st["jprev"] = [z4() for _ in range(3)]
        m = coef[moc]  # (nx, ny, nz, 2 + 7P)
        st["cejsum"][cells] = m[..., 0][cells]
        if a["kind"] == 0:
            st["ceep"][cells] = m[..., 1][cells]
        for p in range(P):
            for q, nm in enumerate(names):
                if nm in st:
                    st[nm][..., p][cells] = m[..., 2 + 7 * p + q][cells]
        return st

    def add_nf2ff(self, nf=3, nt=8, dist=2, batch=3):
        rng = self.rng
        tasks = []
        for face in range(6):
            m, positive = face // 2, face % 2
            s = [dist] * 3
            e = [self.n[a] - dist for a in range(3)]
            c = e[m] if positive else s[m]
            s[m], e[m] = c, c + 1
            tasks.append((s, e))
        self.nf2ff = {"nf": nf, "nt": nt, "tasks": tasks, "batch": batch,
                      "te": rng.standard_normal((nf, nt, 2)),
                      "th": rng.standard_normal((nf, nt, 2))}

    def oracle_nf2ff(self):
        if self.nf2ff is None:
            return None
        nf = self.nf2ff
        offs, total = [], 0
        for f in range(nf["nf"]):
            for face in range(6):
                s, e = nf["tasks"][face]
                npts = (e[0] - s[0]) * (e[1] - s[1]) * (e[2] - s[2])
                for _ in range(4):
                    offs.append(total)
                    total += npts
        out = dict(nf)
        out["acc"] = np.zeros(2 * total)
        out["off"] = np.array(offs, dtype=np.int64)
        return out


def tfsf_source(n, start, steps, theta=0.7, phi=0.4, psi=0.3, shift=12):
    """The oracle's TFSF source (box `start` cells in on every axis, an
    oblique plane wave) for an empty lattice of n cells of 7.5 mm, as the
    dict KernelCase.tfsf takes; the incident grid is started `shift` steps
    late so that the pulse reaches the box within a few steps."""
    from oracle.reference_model import RefSimulation
    from xfdtd_core_b200 import scene as S
    dl = 7.5e-3
    sc = S.Scene(dl=(dl, dl, dl), cfl=0.9, steps=steps + shift, name="tfsf_source")
    sc.objects.append(S.ObjectSpec("domain", S.cube((0.0, 0.0, 0.0),
                                                    tuple(c * dl for c in n)), S.air()))
    tau = dl * 20 / 6e8
    sc.tfsf = S.TFSFSpec(start[0], start[1], start[2], theta, phi, psi,
                         S.Waveform("gaussian", tau, 4.5 * tau))
    r = RefSimulation(sc)
    assert (r.nx, r.ny, r.nz) == tuple(n)
    t = dict(r.tfsf)
    t["e_inc"] = np.ascontiguousarray(t["e_inc"][shift:])
    t["h_inc"] = np.ascontiguousarray(t["h_inc"][shift:])
    t["nt"] = steps
    return t


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
