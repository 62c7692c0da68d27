"""CPU checks of bench.py's plumbing: the reference arm's JSON line, and the
N>1 path (gloo, world size 2): barrier, max-over-ranks timing, rank-0-only
reference arm."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _, pg = bench.dist_setup(world)
    bench.barrier(pg)
    v = bench.max_over_ranks(pg, float(r + 1) * 1.5)
    bench.barrier(pg)
    with open(os.path.join(out, f"r{r}.txt"), "w") as fh:
        fh.write(f"{w} {v}")
    pg.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        w, v = open(tmp_path / f"r{r}.txt").read().split()
        assert int(w) == 2 and float(v) == 3.0


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "boxes", "--grid", "40", "--steps", "4", "--warmup", "3"],
                         capture_output=True,
                         text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "Gcell-updates/s" and line["unit"] == "Gcell/s"
    # the reference's own library where oracle/_ref is built, else the port
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_under_torchrun_rank0_only():
    port = _free_port()
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                          "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                          "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                          "--impl", "reference", "--gpus", "2", "--workload", "boxes", "--grid",
                          "40", "--steps", "3", "--warmup", "3"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["impl"] == "reference"


def test_reference_arm_sphere_workload_counts_its_own_cells():
    """The reference's dielectric-sphere example (63^3): the line names the
    workload and counts the example's cells, not the --grid default."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", "sphere", "--steps", "5", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["config"]["workload"].startswith("dielectric_sphere_63^3")
    assert line["config"]["cells"] == 63 ** 3
    assert "63x63x63" in line["cpu_baseline"]["sample"]
    assert line["value"] > 0
