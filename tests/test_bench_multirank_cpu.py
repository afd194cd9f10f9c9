"""bench.py's multi-rank host logic on CPU: two gloo ranks (torch.distributed), as torchrun
launches them on two GPUs. The whole-job figures take the slowest rank's time and the sum of all
ranks' particle-turns; the reference arm does its work on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    ms = [100.0, 250.0][rank]
    pt = [1000, 3000][rank]
    es = [2.0, 1.5][rank]
    ept = [900, 2900][rank]
    res = bench.combine_ranks(ms, pt, es, ept, world, torch.device("cpu"))
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        assert out[r] == (250.0, 4000.0, 2.0, 3800.0)


def test_reference_arm_nonzero_rank_does_no_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
