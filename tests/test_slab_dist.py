"""The x-slab decomposition (xfdtd_core_b200/slab.py) on CPU: two and three
gloo ranks each run the oracle on their slab of a seeded lattice (random
material classes and curl factors, CPML on all six faces, lumped current
sources; and a lattice with an oblique TFSF plane wave and ADE media cut by
slab as well) and exchange the ghost planes' E_y, E_z after every step; the
owned values gathered on rank 0 equal the one-domain oracle run bit for bit.  The
same with SlabRank (the one-process-per-GPU runner) driving the exchange,
the oracle standing in for each rank's engine.  Plus the planning rules:
cuts keep clear of the x-normal CPML layers, and the cut of the ADE node
lists."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = (30, 9, 11)
SLABS = ((0, True, 3), (0, False, 2), (1, True, 2), (1, False, 3), (2, True, 2), (2, False, 2))
STEPS = 7


def _case(media=False):
    from tests.cases import KernelCase, tfsf_source
    c = KernelCase(n=N, seed=21, slabs=SLABS, field_scale=1e-3 if media else 1.0)
    c.add_lumped(comp=2, s=(8, 4, 4), e=(10, 6, 6), n_steps=STEPS)   # across a ghost region
    c.add_lumped(comp=0, s=(14, 3, 3), e=(17, 5, 5), n_steps=STEPS)  # E_x cells
    if media:
        c.tfsf = tfsf_source(N, (6, 3, 3), STEPS)   # x faces 6 and 24: on different ranks
        c.add_ade(kind=0, n_poles=2, n_mat=2, frac=0.3)
    return c


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out, media):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from tests.cases import KernelCase
    from xfdtd_core_b200 import slab
    dist.init_process_group("gloo", rank=rank, world_size=world)
    case = _case(media)
    parts = slab.plan(N[0], world, x_cpml=(3, 2))
    local = slab.split(case, parts)[rank]
    orc = KernelCase.from_setup(local).oracle()
    plan = slab.exchanges(parts)
    for _ in range(STEPS):
        orc.run(1)
        reqs, bufs = [], []
        for dst, dst_plane, src, src_plane in plan:
            for c in slab.GHOST_COMPONENTS:
                if src == rank:
                    reqs.append(dist.isend(torch.from_numpy(orc.e[c][src_plane].copy()), dst))
                if dst == rank:
                    b = torch.empty(orc.e[c][dst_plane].shape, dtype=torch.float64)
                    reqs.append(dist.irecv(b, src))
                    bufs.append((c, dst_plane, b))
        for r in reqs:
            r.wait()
        for c, plane, b in bufs:
            orc.e[c][plane] = b.numpy()
    got = [None] * world
    dist.all_gather_object(got, [a.copy() for a in orc.e + orc.h])
    if rank == 0:
        fields = slab.gather(parts, got, N)
        np.savez(os.path.join(out, "slab.npz"), *fields)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("media", [False, True], ids=["plain", "tfsf_ade"])
@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_equal_one_domain(tmp_path, world, media):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), media), nprocs=world,
                       start_method="spawn")
    z = np.load(tmp_path / "slab.npz")
    got = [z[f"arr_{c}"] for c in range(6)]
    orc = _case(media).oracle()
    orc.run(STEPS)
    for c, (g, w) in enumerate(zip(got, orc.e + orc.h)):
        assert g.shape == w.shape and np.array_equal(g, w), c


def test_plan_keeps_cuts_clear_of_x_cpml():
    from xfdtd_core_b200 import slab
    parts = slab.plan(100, 4, x_cpml=(10, 10))
    assert [p.own_lo for p in parts] == [0, 25, 50, 75] and parts[-1].own_hi == 100
    assert [(p.lo, p.hi) for p in parts] == [(0, 26), (24, 51), (49, 76), (74, 100)]
    with pytest.raises(ValueError):
        slab.plan(24, 2, x_cpml=(11, 10))  # ghost plane 11 of the cut at 12 is a CPML layer
    ex = slab.exchanges(parts)
    assert (1, 0, 0, 24) in ex and (0, 26, 1, 2) in ex and len(ex) == 6


def test_split_cuts_ade_nodes_and_passes_the_tfsf_offset():
    from xfdtd_core_b200 import slab
    case = _case(media=True)
    parts = slab.plan(N[0], 3, x_cpml=(3, 2))
    local = slab.split(case, parts)
    node, comp = case.ade["node"], case.ade["comp"]
    for p, l in zip(parts, local):
        assert l.tfsf["x_offset"] == p.lo and l.tfsf["box_s"] == case.tfsf["box_s"]
        x = node[:, 0]
        want = np.where(comp == 0, (x >= p.lo) & (x < p.hi), (x > p.lo) & (x < p.hi))
        assert len(l.ade["comp"]) == int(want.sum())
        assert np.array_equal(l.ade["node"][:, 0] + p.lo, x[want])
        assert l.ade["cells"].shape == (p.n,) + N[1:]
    # every owned dispersive node sits in the list of the rank that owns it
    for (i, j, k), c in zip(node, comp):
        owners = [r for r, p in enumerate(parts) if p.own_lo <= i < p.own_hi]
        assert len(owners) == 1
        p, l = parts[owners[0]], local[owners[0]]
        hit = (l.ade["node"] == (i - p.lo, j, k)).all(axis=1) & (l.ade["comp"] == c)
        assert hit.sum() == 1


class _OracleEngine:
    """Stand-in for a slab's engine in SlabRank on CPU: the oracle of the
    slab steps, and plane_copy moves the ghost components of one x-plane
    between the oracle's arrays and the exchange buffer (a (ny+1) x (nz+1)
    segment per component in this stand-in's layout)."""

    def __init__(self, setup):
        from tests.cases import KernelCase
        self.orc = KernelCase.from_setup(setup).oracle()
        self.n = tuple(setup.n)

    def plane_values(self):
        return (self.n[1] + 1) * (self.n[2] + 1)

    def run(self, k):
        self.orc.run(k)

    def plane_copy(self, plane, comps, ptr, into_engine):
        import ctypes
        pv = self.plane_values()
        buf = np.ctypeslib.as_array((ctypes.c_double * (pv * len(comps))).from_address(ptr))
        for q, c in enumerate(comps):
            shape = self.orc.e[c][plane].shape  # a component's plane fits in (ny+1) x (nz+1)
            part = buf[q * pv:q * pv + shape[0] * shape[1]]
            if into_engine:
                self.orc.e[c][plane] = part.reshape(shape)
            else:
                part[:] = self.orc.e[c][plane].ravel()

    def sync(self):
        pass

    def download_fields(self):
        return [a.copy() for a in self.orc.e + self.orc.h]

    def close(self):
        pass


def _rank_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from xfdtd_core_b200 import slab
    dist.init_process_group("gloo", rank=rank, world_size=world)
    slab.make_engine = lambda s, *a, **k: _OracleEngine(s)
    case = _case(media=True)
    parts = slab.plan(N[0], world, x_cpml=(3, 2))
    run = slab.SlabRank(slab.split(case, parts)[rank], parts, rank, device=0, n_steps=STEPS)
    run.step(STEPS)
    fields = run.fields()
    if rank == 0:
        np.savez(os.path.join(out, "rank.npz"), *fields)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_rank_exchange_equals_one_domain(tmp_path, world):
    """SlabRank's exchange (plane_copy into gloo buffers, one
    batch_isend_irecv per step, plane_copy back) with the oracle standing in
    for each rank's engine: the gathered fields equal the one-domain oracle
    bit for bit (oblique TFSF wave and ADE media cut per slab)."""
    import torch.multiprocessing as mp
    mp.start_processes(_rank_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn")
    z = np.load(tmp_path / "rank.npz")
    orc = _case(media=True).oracle()
    orc.run(STEPS)
    for c, w in enumerate(orc.e + orc.h):
        assert np.array_equal(z[f"arr_{c}"], w), c
