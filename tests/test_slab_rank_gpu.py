"""The slab decomposition run by one process per slab (xfdtd_core_b200.slab.SlabRank):
two and three processes, each with its own engine, exchange their ghost
planes' E_y, E_z with torch.distributed after every step (gloo with pinned
host buffers here: every process runs on the one GPU this test has, and no
kernel of one process waits on another's -- the host moves the planes
between the steps; on several GPUs the same class uses NCCL with device
buffers).  The gathered owned values match the one-domain oracle within
1e-12 (FP64), with an oblique TFSF plane wave and ADE media cut per slab."""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = (96, 20, 140)
STEPS = 6
SLABS = ((0, True, 4), (0, False, 3), (1, True, 3), (1, False, 3), (2, True, 3), (2, False, 4))


def _case():
    from tests.cases import KernelCase, tfsf_source
    c = KernelCase(n=N, seed=35, slabs=SLABS, field_scale=1e-3)
    c.tfsf = tfsf_source(N, (9, 4, 9), STEPS)
    c.add_ade(kind=0, n_poles=2, n_mat=2, frac=0.2, margin=5)
    return c


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out, kernel):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from datetime import timedelta
    import torch.distributed as dist
    from xfdtd_core_b200 import slab
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    case = _case()
    parts = slab.plan(N[0], world, x_cpml=(4, 3))
    run = slab.SlabRank(slab.split(case, parts)[rank], parts, rank, device=0, n_steps=STEPS,
                        options={"kernel": kernel})
    run.step(STEPS)
    run.sync()
    fields = run.fields()
    run.close()
    if rank == 0:
        np.savez(os.path.join(out, "rank.npz"), *fields)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("kernel", [0, 7])
@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_on_the_gpu_match_oracle(tmp_path, world, kernel):
    import torch.multiprocessing as mp
    from tests.cases import rel_l2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), kernel), nprocs=world,
                       start_method="spawn")
    z = np.load(tmp_path / "rank.npz")
    got = [z[f"arr_{c}"] for c in range(6)]
    orc = _case().oracle()
    orc.run(STEPS)
    errs = [rel_l2(g, w) for g, w in zip(got, orc.e + orc.h)]
    assert max(errs) <= 1e-12, errs
