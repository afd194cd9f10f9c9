"""bench.py's multi-rank host logic on CPU: two gloo ranks (torch.distributed), as torchrun
launches them on two GPUs. The whole-job figures take the slowest rank's time and the sum of all
ranks' particle-turns; the reference arm does its work on rank 0 only."""
import os
import socket
import subprocess
import sys

import numpy as np
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


# ---- particle sharding and the cross-rank moment sum -----------------------------------------

def _moments(vec, state):
    """Per-turn moment sums of the live particles in the library's layout: n_live, sum vec_i,
    sum vec_i vec_j (i <= j)."""
    alive = state == 1
    v = vec[:, alive]
    out = [float(alive.sum())] + [float(np.sum(v[i])) for i in range(6)]
    out += [float(np.sum(v[i] * v[j])) for i in range(6) for j in range(i, 6)]
    return np.array(out)


def _host_tracker():
    """The device code's host build (test-only) tracking SoA buffers in place, state and beta
    carried from call to call."""
    import ctypes
    import importlib
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_hostcheck_cpu import HC
    abi = importlib.import_module("bmad-ecosystem_b200.abi")
    if not os.path.exists(HC):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "bmad-ecosystem_b200", "csrc"), "hostcheck-lib"])
    hc = ctypes.CDLL(HC)

    def track(eles, p, vec, beta, state, n_turns):
        arr = abi.element_array(eles)
        b = abi.Bunch(vec.shape[1], vec.ctypes.data, beta.ctypes.data, None, state.ctypes.data, None, None, None)
        assert hc.bmadgpu_hostcheck_track(arr, len(arr), ctypes.byref(p), ctypes.byref(b), n_turns) == 0
    return track


def _start(eles, p, n):
    import importlib
    rings = importlib.import_module("bmad-ecosystem_b200.rings")
    vec = np.ascontiguousarray(rings.matched_gaussian(eles, n, seed=17, scale=10.0))   # wide: some are lost
    pc = p.p0c * (1 + vec[5])
    return vec, np.ascontiguousarray(pc / np.sqrt(pc * pc + p.mass ** 2)), np.ones(n, np.int32)


def _shard_rank(rank, world, port, out, n, n_turns):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import importlib
    lib = importlib.import_module("bmad-ecosystem_b200.lib")
    rings = importlib.import_module("bmad-ecosystem_b200.rings")
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    track = _host_tracker()
    eles, p = rings.ring(50)
    vec, beta, state = _start(eles, p, n)
    a, b = lib.shard(n, rank, world)
    mine, mb, ms = np.ascontiguousarray(vec[:, a:b]), beta[a:b].copy(), state[a:b].copy()
    mom = np.zeros((n_turns, 28))
    for t in range(n_turns):      # one turn per call, the moments after each turn
        track(eles, p, mine, mb, ms, 1)
        mom[t] = _moments(mine, ms)
    total = lib.allreduce_moments(mom)
    out[rank] = (a, b, mine, ms, mom, total)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_tracking_and_moment_allreduce_two_gloo_ranks():
    """Two ranks each track their shard of one bunch (the device code's host build) and add their
    per-turn moment sums with one all_reduce: every particle and both ranks' totals equal the
    one-rank computation bit for bit (two partial sums, added once)."""
    import importlib
    n, n_turns = 601, 6
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, out, n, n_turns)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    rings = importlib.import_module("bmad-ecosystem_b200.rings")
    eles, p = rings.ring(50)
    vec, beta, state = _start(eles, p, n)
    _host_tracker()(eles, p, vec, beta, state, n_turns)     # one rank, all particles, all turns at once
    ref = dict(vec=vec, state=state)
    assert (ref["state"] != 1).sum() > 10
    (a0, b0, v0, s0, m0, t0), (a1, b1, v1, s1, m1, t1) = out[0], out[1]
    assert (a0, b0, a1, b1) == (0, 301, 301, 601)
    assert np.array_equal(np.concatenate([v0, v1], axis=1), ref["vec"])
    assert np.array_equal(np.concatenate([s0, s1]), ref["state"])
    assert np.array_equal(t0, m0 + m1) and np.array_equal(t1, m0 + m1)
    whole = _moments(ref["vec"], ref["state"])
    assert np.allclose(t0[-1], whole, rtol=1e-12, atol=0)


def test_shard_ranges_cover_the_bunch():
    import importlib
    lib = importlib.import_module("bmad-ecosystem_b200.lib")
    for n in (0, 1, 7, 1000, 1048576):
        for world in (1, 2, 3, 8):
            r = [lib.shard(n, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
            assert max(b - a for a, b in r) - min(b - a for a, b in r) <= 1
