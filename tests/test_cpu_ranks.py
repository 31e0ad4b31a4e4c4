"""Multi-process plumbing of bench.py on the CPU: world size 2 over gloo.

bench.py runs one process per GPU; each renders its own replica and rank 0 reports the max
device time over ranks and the sum of rays. These tests run the same Ranks helper over gloo
with two CPU processes, and check that the reference arm does nothing on ranks other than 0.
"""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    ranks = bench.Ranks.init("gloo", rank, timeout_s=60)
    ranks.barrier()
    ms = ranks.max(10.0 * (rank + 1))      # device time of this rank
    rays = ranks.sum(1000.0 * (rank + 1))  # rays of this rank
    ranks.barrier()
    with open(f"{out_path}.{rank}", "w") as f:
        f.write(f"{ms} {rays}\n")
    ranks.pg.destroy_process_group()


def test_max_and_sum_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r")
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        ms, rays = map(float, open(f"{out}.{r}").read().split())
        assert ms == 20.0 and rays == 3000.0


def test_single_process_ranks_are_identity():
    sys.path.insert(0, ROOT)
    import bench

    ranks = bench.Ranks(None, None)
    ranks.barrier()
    assert ranks.max(3.5) == 3.5 and ranks.sum(7.0) == 7.0


def test_reference_arm_is_silent_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
