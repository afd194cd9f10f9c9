"""Serving (bmadgpu_server_*): continuous batching of tracking jobs of different lattices,
particle counts and turn counts, submitted while others are on the GPU.

The central check: each job's result in the mix is the same as the job run alone -- through the
plain path (bmadgpu_track_bunch with the job's turns per round as turns per launch) and through a
server holding only that job -- bit for bit in every coordinate, state, loss record and time.
Also: admission never exceeds the resident arena; oversize jobs are refused; latency and
throughput statistics; FIFO and shortest-remaining-work policies; wait time-outs."""
import importlib
import time

import numpy as np
import pytest

from conftest import load_abi

pytestmark = pytest.mark.gpu
lib = importlib.import_module("bmad-ecosystem_b200.lib")
rings = importlib.import_module("bmad-ecosystem_b200.rings")
abi = load_abi()

FIELDS = ("vec", "beta", "state", "ix_ele", "ix_turn", "location", "t")


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def make_jobs(specs):
    """specs: (n_cells, seed, n_particles, n_turns, kind) -> [(elements, param, vec, t, n_turns)]."""
    out = []
    for n_cells, seed, n, turns, kind in specs:
        eles, param = rings.perturbed_ring(n_cells, seed=seed)
        if kind == "gauss":
            vec = rings.matched_gaussian(eles, n, seed=seed, scale=2.0)
        else:
            vec = rings.da_grid(n, r_max=0.02)
        t = np.random.default_rng(seed).normal(0.0, 1e-9, n)
        out.append((eles, param, vec, t, turns))
    return out


SPECS = [(3, 1, 300, 17, "grid"), (6, 2, 2000, 40, "gauss"), (10, 3, 1, 5, "gauss"), (4, 4, 5000, 23, "grid"),
         (8, 5, 77, 64, "gauss"), (5, 6, 1024, 9, "grid"), (12, 7, 0, 10, "gauss"), (2, 8, 640, 0, "grid")]


def per_round(eles, element_steps):
    return max(1, element_steps // len(eles))


def result(b):
    return {f: None if getattr(b, f) is None else np.array(getattr(b, f)) for f in FIELDS}


def plain_alone(ctx, eles, param, vec, t, turns, tpl):
    ctx.set_tuning(block=128, ctas_per_sm=0, stage_smem=1, turns_per_launch=tpl, compact=1)
    b = lib.HostBunch.from_vec(vec, param, t=t)
    if b.n and turns:
        lat = lib.Lattice(ctx, eles, param)
        lib.track_bunch(ctx, lat, b, n_turns=turns)
    ctx.set_tuning(block=128, ctas_per_sm=0, stage_smem=1, turns_per_launch=0, compact=0)
    return result(b)


def assert_same(a, b, tag):
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), "%s: field %s differs" % (tag, f)


@pytest.mark.parametrize("policy", [lib.SERVE_SRPT, lib.SERVE_FIFO])
def test_each_result_same_alone_and_in_mix(ctx, policy):
    steps = 120
    jobs = make_jobs(SPECS)
    srv = lib.Server(ctx, element_steps=steps, policy=policy, target_live=4000)
    lats, bunches, ids = [], [], []
    for k, (eles, p, vec, t, turns) in enumerate(jobs):
        lat = lib.Lattice(ctx, eles, p)
        b = lib.PinnedBunch(vec, lib.HostBunch.from_vec(vec, p).beta, t=t)
        lats.append(lat)
        bunches.append(b)
        ids.append(srv.submit(lat, b, turns))
        if k % 3 == 1:
            time.sleep(0.01)   # later jobs arrive while earlier ones are on the GPU
    srv.wait(-1, timeout=300)
    st = srv.stats()
    assert st["jobs_done"] == len(jobs)
    infos = [srv.job(i) for i in ids]
    srv.close()
    total_pt = 0
    for k, ((eles, p, vec, t, turns), b, info) in enumerate(zip(jobs, bunches, infos)):
        assert info["status"] == lib.JOB_DONE
        got = result(b)
        want = plain_alone(ctx, eles, p, vec, t, turns, per_round(eles, steps))
        assert_same(got, want, "job %d vs plain" % k)
        total_pt += info["particle_turns"]
        if b.n and turns:
            assert 0 <= info["t_submit"] <= info["t_admit"] <= info["t_done"]
    assert total_pt == st["particle_turns"]
    assert st["latency_p50_s"] <= st["latency_p99_s"] <= st["latency_max_s"]

    # the same jobs, each alone on a fresh server
    for k in (0, 3, 4):
        eles, p, vec, t, turns = jobs[k]
        srv = lib.Server(ctx, element_steps=steps, policy=policy)
        lat = lib.Lattice(ctx, eles, p)
        b = lib.PinnedBunch(vec, lib.HostBunch.from_vec(vec, p).beta, t=t)
        srv.wait(srv.submit(lat, b, turns), timeout=120)
        srv.close()
        assert_same(result(b), result(bunches[k]), "job %d alone vs in the mix" % k)


def test_admission_bounded_by_arena(ctx):
    cap = 5000
    srv = lib.Server(ctx, max_particles=cap, element_steps=200)
    eles, p = rings.perturbed_ring(4, seed=9)
    lat = lib.Lattice(ctx, eles, p)
    big = lib.HostBunch.from_vec(rings.matched_gaussian(eles, cap + 1, seed=1), p)
    with pytest.raises(lib.BmadGpuError) as ex:
        srv.submit(lat, big, 5)
    assert ex.value.code == abi.ENOMEM
    bunches = [lib.HostBunch.from_vec(rings.matched_gaussian(eles, 3000, seed=s), p) for s in range(4)]
    ids = [srv.submit(lat, b, 30) for b in bunches]
    srv.wait(-1, timeout=300)
    st = srv.stats()
    assert st["capacity"] == cap
    assert st["peak_resident"] <= cap
    assert st["jobs_done"] == 4
    assert st["peak_resident"] == 3000   # two 3000-particle jobs never fit together
    assert all(srv.job(i)["status"] == lib.JOB_DONE for i in ids)
    srv.close()
    want = plain_alone(ctx, eles, p, rings.matched_gaussian(eles, 3000, seed=0), None, 30, per_round(eles, 200))
    assert np.array_equal(bunches[0].vec, want["vec"])


def test_wait_timeout_and_trivial_jobs(ctx):
    srv = lib.Server(ctx, element_steps=64)
    eles, p = rings.perturbed_ring(20, seed=3)
    lat = lib.Lattice(ctx, eles, p)
    b = lib.HostBunch.from_vec(rings.matched_gaussian(eles, 20000, seed=4), p)
    jid = srv.submit(lat, b, 400)
    with pytest.raises(lib.BmadGpuError) as ex:
        srv.wait(jid, timeout=1e-4)
    assert ex.value.code == abi.ETIMEDOUT
    empty = lib.HostBunch(np.zeros((6, 0)), np.zeros(0))
    j0 = srv.submit(lat, empty, 10)
    assert srv.job(j0)["status"] == lib.JOB_DONE
    srv.wait(jid, timeout=300)
    assert srv.job(jid)["status"] == lib.JOB_DONE
    with pytest.raises(lib.BmadGpuError) as ex:
        srv.job(12345)
    assert ex.value.code == abi.ENOTFOUND
    srv.close()


def test_destroy_cancels_queued_jobs(ctx):
    srv = lib.Server(ctx, max_particles=2000, element_steps=64)
    eles, p = rings.perturbed_ring(10, seed=5)
    lat = lib.Lattice(ctx, eles, p)
    bunches = [lib.HostBunch.from_vec(rings.matched_gaussian(eles, 2000, seed=s), p) for s in range(3)]
    ids = [srv.submit(lat, b, 50) for b in bunches]
    srv.close()   # the resident job finishes; the queued ones are cancelled
    # no exception, no hang; the library has released everything
    assert len(ids) == 3
