"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the
max-over-ranks timing reduction, and the reference arm under torchrun
(rank 0 prints one JSON line, the other rank exits 0 without work, and the
arm loads none of the repository's native libraries)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.dist_max(dist, 1.5 + rank)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_dist_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_dist_max_without_group_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert bench.dist_max(None, 3.25) == 3.25


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--grid", "32"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=580, cwd=REPO, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["higher_is_better"] is False
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["value"] > 0
    # the reference arm runs the CPU port only: none of this repository's native code is mapped
    assert d["native_libs_loaded"] == []
    assert d["config"]["n"] == 32 and d["iterations"] > 0
