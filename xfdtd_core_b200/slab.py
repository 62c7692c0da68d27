"""Slab decomposition of one lattice along x over several engines (GPUs).

The reference decomposes its grid over MPI ranks in slabs with an overlap
and exchanges a halo after every step (src/simulation/simulation.cpp:530-591,
src/domain/domain.cpp:237-279, src/parallel/mpi_support.cpp:98-229).  Here
rank r owns the cells [c_r, c_{r+1}) of the global x range and runs an
ordinary engine on the local lattice of cells [a_r, b_r) = [c_r - 1, c_{r+1}
+ 1) (no extra cell at the global faces): one ghost cell on each interior
side.  One time step of the local engine then leaves every value of its
lattice exact except E_y and E_z on the two ghost planes a_r and b_r, which
the engine treats as lattice boundaries and does not update:

* H_y, H_z of a cell need E on the two planes around it, H_x of a plane
  needs E in that plane: all local, exact when the ghost planes held the
  exact E at the start of the step;
* E_x of a cell needs H of that cell only; E_y, E_z of the interior planes
  a_r + 1 .. b_r - 1 need H_y, H_z of the cells either side: all local.
  (H_x on the high ghost plane is not updated either; only the ghost planes'
  own E reads it.)

So after every step each rank receives E_y, E_z of its ghost plane a_r from
rank r - 1, where that plane is interior, and of b_r from rank r + 1: two
tangential components of one plane per neighbour and step, the dual of the
reference's H halo.  Values in the ghost cells (E_x, H_y, H_z, ADE and CPML
state there) are computed by both neighbours from the same inputs and agree
bit for bit.  The x-normal CPML slabs stay whole on the first and last rank:
cuts keep the ghost cells and planes clear of their layers.  y- and
z-normal slabs, materials, curl factors, fields and lumped sources are cut
by intersection with each local lattice (sources in a ghost region run on
both ranks, which keeps the ghost values exact).  A TFSF source is cut the
same way: each engine takes the global source and its x offset
(xfd_set_tfsf_slab), which keeps only the face passes' nodes of its local
lattice (the reference cuts TFSF3D by its domain, src/waveform_source/
tfsf_3d.cpp:21-33).  ADE media are cut by node: every dispersive E node of
the local lattice, ghost cells included, except E_y, E_z on a ghost or
boundary plane (values the exchange overwrites, and that no update of an
owned value reads).  NF2FF surfaces are not split here: lattices with one run
on one engine.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# Field component -> axis of its x index: E_x, H_y, H_z live on cells (nx
# values), E_y, E_z, H_x on node planes (nx + 1 values).
ON_CELLS = (True, False, False, False, True, True)
GHOST_COMPONENTS = (1, 2)  # E_y, E_z


@dataclass
class SlabPart:
    rank: int
    own_lo: int  # first owned cell (and node plane)
    own_hi: int  # one past the last owned cell; the last rank also owns plane nx
    lo: int      # first cell of the local lattice (own_lo - 1 except on rank 0)
    hi: int      # one past its last cell (own_hi + 1 except on the last rank)

    @property
    def n(self) -> int:
        return self.hi - self.lo


def plan(nx: int, ranks: int, x_cpml: Tuple[int, int] = (0, 0)) -> List[SlabPart]:
    """Cuts of nx cells into `ranks` slabs of nearly equal size.  x_cpml:
    thicknesses of the x-normal CPML slabs at the low and high face; every
    cut c keeps its ghost planes c - 1 .. c + 1 clear of their layers
    (E layers 1 .. lo, H layers 0 .. lo-1 at the low face; from nx - hi up
    at the high face), else ValueError."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    cuts = [round(r * nx / ranks) for r in range(ranks + 1)]
    lo_t, hi_t = x_cpml
    for c in cuts[1:-1]:
        if c - 1 <= lo_t or c + 1 >= nx - hi_t:
            raise ValueError(f"cut at cell {c} meets an x-normal CPML slab "
                             f"(thickness {lo_t} / {hi_t} of {nx} cells)")
    if any(b - a < 2 for a, b in zip(cuts, cuts[1:])):
        raise ValueError("slabs of fewer than two cells")
    parts = []
    for r in range(ranks):
        a = cuts[r] - (1 if r > 0 else 0)
        b = cuts[r + 1] + (1 if r < ranks - 1 else 0)
        parts.append(SlabPart(r, cuts[r], cuts[r + 1], a, b))
    return parts


def _x_range(part: SlabPart, comp6: int) -> slice:
    """Local x index range of a component in global indices."""
    return slice(part.lo, part.hi if ON_CELLS[comp6] else part.hi + 1)


@dataclass
class LocalSetup:
    """Engine inputs of one slab: the arrays of xfd_set_material_classes,
    xfd_set_curl_factors, xfd_add_cpml, xfd_add_current_source and
    xfd_upload_fields over the local lattice."""
    n: Tuple[int, int, int]
    table: np.ndarray
    lattice_class: np.ndarray
    fe: List[np.ndarray]
    fh: List[np.ndarray]
    slabs: List[Dict]
    lumped: List[Dict]
    fields: List[np.ndarray]
    tfsf: Optional[Dict] = None  # the global source plus "x_offset"
    ade: Optional[Dict] = None   # the local dispersive nodes


def split(setup, parts: Sequence[SlabPart]) -> List[LocalSetup]:
    """Cuts a lattice set-up (attributes n, table, lattice_class, fe, fh,
    slabs, lumped, fields; optional tfsf and ade -- the dicts of
    tests.cases.KernelCase -- and nf2ff, which must be None) into the local
    set-ups of `parts`."""
    if getattr(setup, "nf2ff", None):
        raise ValueError("nf2ff is not split across slabs")
    tfsf = getattr(setup, "tfsf", None)
    ade = getattr(setup, "ade", None)
    nx, ny, nz = setup.n
    out = []
    for p in parts:
        a, b = p.lo, p.hi
        slabs = []
        for s in setup.slabs:
            if s["m"] != 0:
                slabs.append(dict(s))
                continue
            # whole x slab on the rank that holds its layers, shifted to local planes
            first = min(s["e_start"], s["h_start"])
            last = max(s["e_start"], s["h_start"]) + s["n"]
            if first >= a and last <= b + 1:
                q = dict(s)
                q["e_start"] = s["e_start"] - a
                q["h_start"] = s["h_start"] - a
                slabs.append(q)
            elif first < b + 1 and last > a:
                raise ValueError("an x-normal CPML slab crosses a slab cut")
        lumped = []
        for l in setup.lumped:
            c = l["comp"]
            hi_x = b if ON_CELLS[c] else b + 1
            s0, e0 = max(l["s"][0], a), min(l["e"][0], hi_x)
            if s0 >= e0:
                continue
            q = dict(l)
            q["s"] = [s0 - a, l["s"][1], l["s"][2]]
            q["e"] = [e0 - a, l["e"][1], l["e"][2]]
            q["coff"] = np.ascontiguousarray(l["coff"][s0 - l["s"][0]:e0 - l["s"][0]])
            lumped.append(q)
        fields = [np.ascontiguousarray(f[_x_range(p, c)]) for c, f in enumerate(setup.fields)]
        ltfsf = None
        if tfsf:
            ltfsf = dict(tfsf)
            ltfsf["x_offset"] = a
        lade = None
        if ade:
            node = np.asarray(ade["node"]).reshape(-1, 3)
            comp = np.asarray(ade["comp"])
            x = node[:, 0]
            # E_x on cells [a, b); E_y, E_z on the planes strictly inside (a, b)
            keep = np.where(comp == 0, (x >= a) & (x < b), (x > a) & (x < b))
            local = node[keep].copy()
            local[:, 0] -= a
            lade = {k: v for k, v in ade.items()
                    if k not in ("node", "comp", "material", "cells", "mat_of_cell")}
            lade.update(node=np.ascontiguousarray(local, dtype=np.int32),
                        comp=np.ascontiguousarray(comp[keep]),
                        material=np.ascontiguousarray(np.asarray(ade["material"])[keep]))
            for key in ("cells", "mat_of_cell"):  # per-cell form, where given
                if key in ade:
                    lade[key] = np.ascontiguousarray(ade[key][a:b])
        out.append(LocalSetup(
            n=(b - a, ny, nz), table=setup.table,
            lattice_class=np.ascontiguousarray(setup.lattice_class[a:b + 1]),
            fe=[np.ascontiguousarray(setup.fe[0][a:b + 1])] + [setup.fe[1], setup.fe[2]],
            fh=[np.ascontiguousarray(setup.fh[0][a:b])] + [setup.fh[1], setup.fh[2]],
            slabs=slabs, lumped=lumped, fields=fields, tfsf=ltfsf, ade=lade))
    return out


def exchanges(parts: Sequence[SlabPart]) -> List[Tuple[int, int, int, int]]:
    """The ghost-plane copies after every step: (destination rank, its local
    plane, source rank, its local plane), for E_y and E_z alike."""
    out = []
    for r, p in enumerate(parts):
        if r > 0:
            q = parts[r - 1]
            out.append((r, 0, r - 1, p.lo - q.lo))
        if r < len(parts) - 1:
            q = parts[r + 1]
            out.append((r, p.n, r + 1, p.hi - q.lo))
    return out


def owned(part: SlabPart, comp6: int, nx: int) -> Tuple[slice, slice]:
    """(global, local) x index ranges of the values a rank owns: its cells,
    or its node planes [own_lo, own_hi) -- the last rank also plane nx."""
    hi = part.own_hi
    if not ON_CELLS[comp6] and part.own_hi == nx:
        hi = nx + 1
    return slice(part.own_lo, hi), slice(part.own_lo - part.lo, hi - part.lo)


def gather(parts: Sequence[SlabPart], local_fields: Sequence[Sequence[np.ndarray]],
           n: Tuple[int, int, int]) -> List[np.ndarray]:
    """The global fields from every rank's owned values."""
    from xfdtd_core_b200.engine import comp_shape
    out = [np.empty(comp_shape(n, c), dtype=local_fields[0][c].dtype) for c in range(6)]
    for p, f in zip(parts, local_fields):
        for c in range(6):
            g, l = owned(p, c, n[0])
            out[c][g] = f[c][l]
    return out


# ------------------------------------------------------------ engine runners
def make_engine(s: LocalSetup, device: int = 0, precision: int = 0, n_steps: int = 1,
                options: Optional[Dict[str, int]] = None):
    """An engine over one slab's local set-up."""
    from xfdtd_core_b200.engine import Engine
    e = Engine(*s.n, precision=precision, n_steps=n_steps, dt=1.0, device=device)
    for k, v in (options or {}).items():
        e.set_option(k, v)
    e.set_material_classes(s.table, s.lattice_class)
    e.set_curl_factors(s.fe, s.fh)
    for sl in s.slabs:
        e.add_cpml(sl["m"], sl["neg"], sl["n"], sl["e_start"], sl["h_start"], sl["a_e"],
                   sl["b_e"], sl["a_h"], sl["b_h"])
    for l in s.lumped:
        e.add_current_source(l["comp"], l["s"], l["e"], l["coff"], l["wave"])
    if s.tfsf is not None:
        t = s.tfsf
        e.set_tfsf(t["box_s"], t["box_e"], t["e_inc"], t["h_inc"], t["p_int"], t["p_half"],
                   t["ca"], t["cb"], t["te"], t["th"], x_offset=t["x_offset"])
    if s.ade is not None and len(s.ade["comp"]):
        a = s.ade
        e.set_ade(a["kind"], a["np"], a["mat_coeff"], a["comp"], a["node"], a["material"])
    e.upload_fields([f.astype(e.dtype) for f in s.fields])
    return e


class SlabEngines:
    """One engine per slab in this process (each on its own device, or all on
    one), stepped together: every step runs each engine one step, then copies
    the ghost planes' E_y, E_z with xfd_halo_copy (device to device, a peer
    copy between devices; ordered on the engines' streams, so no engine
    starts its next step before its ghost planes hold the neighbours' values
    or overwrites a plane a neighbour is still copying)."""

    def __init__(self, setups: Sequence[LocalSetup], parts: Sequence[SlabPart],
                 devices: Optional[Sequence[int]] = None, precision: int = 0,
                 n_steps: int = 1, options: Optional[Dict[str, int]] = None):
        self.parts = list(parts)
        self.devices = list(devices) if devices is not None else [0] * len(parts)
        self.engines = [make_engine(s, dev, precision, n_steps, options)
                        for s, dev in zip(setups, self.devices)]
        self.plan = exchanges(self.parts)

    def step(self, n: int = 1):
        for _ in range(n):
            for e in self.engines:
                e.run(1)
            for dst, dst_plane, src, src_plane in self.plan:
                self.engines[dst].halo_copy_from(dst_plane, self.engines[src], src_plane,
                                                 GHOST_COMPONENTS)

    def sync(self):
        for e in self.engines:
            e.sync()

    def fields(self) -> List[np.ndarray]:
        n = (self.parts[-1].own_hi,) + tuple(self.engines[0].n[1:])
        return gather(self.parts, [e.download_fields() for e in self.engines], n)

    def close(self):
        for e in self.engines:
            e.close()


class SlabRank:
    """One rank of a slab decomposition run by one process per GPU under
    torch.distributed (the form for several GPUs of one node: the reference
    runs one MPI process per domain).  The rank holds the engine of its slab;
    after every step the ghost planes' E_y, E_z move to the neighbours with
    torch.distributed point-to-point calls, grouped in one batch_isend_irecv
    so that every rank posts the same calls in the same order.  On an NCCL
    process group the buffers are tensors on this rank's GPU, and the planes
    go GPU to GPU (through NVLink between peers; no library kernel ever reads
    another GPU's memory); on gloo they are pinned host tensors.  The engine's
    stream and the transfer meet on the host: the planes are copied out and
    the stream synchronised before the sends, and copied in after the
    receives completed."""

    def __init__(self, setup: LocalSetup, parts: Sequence[SlabPart], rank: int, device: int = 0,
                 group=None, precision: int = 0, n_steps: int = 1,
                 options: Optional[Dict[str, int]] = None):
        import torch
        import torch.distributed as dist
        self.parts, self.rank, self.group = list(parts), rank, group
        self.device = device
        self.engine = make_engine(setup, device, precision, n_steps, options)
        self.plan = exchanges(self.parts)
        self.on_device = dist.get_backend(group) == "nccl"
        dtype = torch.float64 if precision == 0 else torch.float32
        size = len(GHOST_COMPONENTS) * self.engine.plane_values()

        def buf():
            if self.on_device:
                return torch.empty(size, dtype=dtype, device=torch.device("cuda", device))
            t = torch.empty(size, dtype=dtype)
            return t.pin_memory() if torch.cuda.is_available() else t

        self.send = {(d, sp): buf() for d, dp, s, sp in self.plan if s == rank}
        self.recv = {(s, dp): buf() for d, dp, s, sp in self.plan if d == rank}

    def step(self, n: int = 1):
        import torch
        import torch.distributed as dist
        for _ in range(n):
            self.engine.run(1)
            for d, dp, s, sp in self.plan:
                if s == self.rank:
                    self.engine.plane_copy(sp, GHOST_COMPONENTS, self.send[(d, sp)].data_ptr(),
                                           into_engine=False)
            self.engine.sync()
            ops = []
            for d, dp, s, sp in self.plan:  # the same list, in the same order, on every rank
                if s == self.rank:
                    ops.append(dist.P2POp(dist.isend, self.send[(d, sp)], d, self.group))
                if d == self.rank:
                    ops.append(dist.P2POp(dist.irecv, self.recv[(s, dp)], s, self.group))
            if ops:
                for r in dist.batch_isend_irecv(ops):
                    r.wait()
            if self.on_device:
                torch.cuda.synchronize(self.device)
            for d, dp, s, sp in self.plan:
                if d == self.rank:
                    self.engine.plane_copy(dp, GHOST_COMPONENTS, self.recv[(s, dp)].data_ptr(),
                                           into_engine=True)

    def sync(self):
        self.engine.sync()

    def fields(self) -> List[np.ndarray]:
        """The global fields, on every rank (the owned values of all ranks)."""
        import torch.distributed as dist
        local = self.engine.download_fields()
        got = [None] * len(self.parts)
        dist.all_gather_object(got, local, group=self.group)
        n = (self.parts[-1].own_hi,) + tuple(self.engine.n[1:])
        return gather(self.parts, got, n)

    def close(self):
        self.engine.close()
