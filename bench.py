#!/usr/bin/env python
"""Benchmark: particle-turns/s of FP64 multi-turn bunch tracking on one or more B200s.

Workload (default "ring200"): the 200-cell FODO ring with random b3..b10 sextupole multipoles
(seed 1) and sbend edge fringes, 1,048,576 particles per GPU in a 3-sigma matched Gaussian,
tracked in FP64 through all 1801 elements per turn (the plain large configuration of the
benchmark suite). A step is `--turns-per-step` turns of the whole bunch; the bunch keeps its
state from step to step, as long-term tracking does. "ring50" is the 50-cell ring with 10,000
particles (the small configuration).

ours (default): the sm_100a kernel through the C-ABI. `value` is device-resident throughput
(particle-turns actually tracked / kernel time, CUDA events on the library's stream, L2 flushed
between steps); `e2e` is the same metric through the host-pointer API, host<->device copies of
the whole bunch included every step.
--impl reference: the reference algorithm's CPU implementation (the C++ oracle restating the
Fortran track1_bunch path, OpenMP over particles) on the host cores, bounded samples.

The default line (ring200 on one GPU) also carries the benchmark's other headline figures as
sub-records, each timed in its own region: "correctly_rounded" (the same ring200 workload with
libbmadgpu_cr.so, the build whose transcendentals are correctly rounded and whose results are
bit-identical to the oracle run with a correctly rounded libm), "batched" (the batch256 job, one step, against the
plain kernel on 8 sampled variants), "served" (the first 200 jobs of the request stream, p50/p99
latency, against the plain kernel on 8 sampled jobs) and "adjoint" (gradients/s); --no-extras
leaves them out.

Further workloads (one JSON line each, same keys):
  batch256  256 perturbed 50-cell rings (strengths, offsets, tilts per variant seed), each with a
            dynamic-aperture grid of log-uniform [1024, 65536] particles, 2048 turns; a step is the
            whole job from the initial grids through the batched path (one persistent launch per
            batch of turns, CUDA-graph replay, autotuned). Beside it: the plain kernel run variant
            by variant on a random sample of the variants (ratio estimate of its aggregate).
  serve     the Poisson request stream of tracking jobs (mean gap 5 ms; 50/100/200/400-cell
            perturbed rings; log-uniform [256, 262144] particles and [64, 4096] turns; Gaussian or
            frequency-map grid), the first --jobs jobs, through the continuous-batching server from
            host memory; p50/p99 latency; beside it the plain kernel on a sample of the same jobs.
  adjoint   d(loss)/d(100 quadrupole k1, 100 sextupole k2) on the 50-cell ring, 4096 particles,
            256 turns, checkpoints every 16 turns; a step is one gradient.
  kinds     the plain kernel's cost per element kind: lattices of 1800 copies of each kind of
            ring200 (drift, quadrupole, exact bend with and without Hwang edges, sextupole with and
            without b3..b10) and ring200 itself, 1,048,576 small-amplitude particles, one turn per
            step at the context's default launch shape; ns per particle-element.

Multi-GPU: one process per GPU (torchrun); each rank tracks its own bunch (particles never
interact: weak scaling, no collective on the data path); the timing is the max over ranks.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import importlib  # noqa: E402

import numpy as np  # noqa: E402

PKG = "bmad-ecosystem_b200"
abi = importlib.import_module(PKG + ".abi")
rings = importlib.import_module(PKG + ".rings")

METRIC = "particle-turns/s (FP64, plain kernel)"
UNIT = "particle-turns/s"


def workload(name, rank):
    if name == "ring200":
        eles, p = rings.ring(200, fringe=True, multipole_sigma=1e-4, multipole_seed=1)
        n, scale = 1048576, 3.0
    elif name == "ring50":
        eles, p = rings.ring(50)
        n, scale = 10000, 1.0
    else:
        raise SystemExit("unknown workload " + name)
    return eles, p, n, scale


def config_dict(args, n, n_ele):
    return {"workload": "%s: %d-element ring, %d particles/GPU, %d turns/step, FP64" % (
        args.workload, n_ele, n, args.turns_per_step),
        "particles_per_gpu": n, "elements": n_ele, "turns_per_step": args.turns_per_step,
        "l2": "flushed between steps (256 MiB write)", "parallelism": "particle sharding, %d rank(s)" % args.gpus}


# ---------------------------------------------------------------------------------------------
# CPU: the oracle (checker / CPU baseline only)

def load_oracle():
    path = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(path):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    lib.oracle_track_ring.argtypes = [P(abi.Element), ctypes.c_int32, P(abi.Param), P(abi.Bunch), ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_int32, P(ctypes.c_double)]
    lib.oracle_max_threads.restype = ctypes.c_int32
    return lib


def oracle_rate(eles, p, vec0, n_turns, threads):
    """Particle-turns/s of the oracle on vec0[6, n] for n_turns."""
    lib = load_oracle()
    arr = abi.element_array(eles)
    vec = np.array(vec0, copy=True)
    n = vec.shape[1]
    pc = p.p0c * (1 + vec[5])
    beta = np.ascontiguousarray(pc / np.sqrt(pc * pc + p.mass ** 2))
    st = np.ones(n, np.int32)
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, None, st.ctypes.data, None, None, None)
    t0 = time.perf_counter()
    err = lib.oracle_track_ring(arr, len(arr), ctypes.byref(p), ctypes.byref(b), 0, n_turns, threads, None)
    dt = time.perf_counter() - t0
    assert err == 0
    return n * n_turns / dt, dt


def cpu_baseline(eles, p, scale, budget_s=12.0):
    """The oracle on the host cores: a probe sizes one sample to about budget_s of CPU work."""
    threads = load_oracle().oracle_max_threads()
    vec = rings.matched_gaussian(eles, 512, seed=123, scale=scale)
    rate, _ = oracle_rate(eles, p, vec, 1, threads)
    n = int(min(max(512, rate * budget_s), 1 << 18))
    vec = rings.matched_gaussian(eles, n, seed=123, scale=scale)
    rate, dt = oracle_rate(eles, p, vec, 1, threads)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d particles x 1 turn of the same ring (%.1f s), C++ oracle restating the Fortran "
                      "track1_bunch path, OpenMP %d threads" % (n, dt, threads)}


# ---------------------------------------------------------------------------------------------
# GPU helpers

class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def op_count(eles, p, scale):
    """Algorithmic FP64 ops per particle-turn of the device code (op-counting host build of the
    same source): add/sub, mul, div, sqrt and transcendental calls each count one."""
    path = os.path.join(ROOT, PKG, "_build", "libbmadgpu_hostcount.so")
    if not os.path.exists(path):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, PKG, "csrc"), "hostcheck-lib"])
    lc = ctypes.CDLL(path)
    vec = np.array(rings.matched_gaussian(eles, 256, seed=7, scale=scale), copy=True)
    n = vec.shape[1]
    pc = p.p0c * (1 + vec[5])
    beta = np.ascontiguousarray(pc / np.sqrt(pc * pc + p.mass ** 2))
    st = np.ones(n, np.int32)
    b = abi.Bunch(n, vec.ctypes.data, beta.ctypes.data, None, st.ctypes.data, None, None, None)
    cnt = (ctypes.c_double * 6)()
    arr = abi.element_array(eles)
    assert lc.bmadgpu_hostcheck_count_ops(arr, len(arr), ctypes.byref(p), ctypes.byref(b), 2, cnt) == 0
    per = [cnt[i] / cnt[5] for i in range(5)]
    return sum(per), dict(zip(["add", "mul", "div", "sqrt", "transcendental"], per))


def combine_ranks(total_ms, total_pt, e2e_s, e2e_pt, world, dev):
    """Whole-job figures over ranks: the slowest rank's times (max) and every rank's
    particle-turns (sum); each rank tracks its own particles (weak scaling)."""
    import torch
    import torch.distributed as dist
    vals = torch.tensor([total_ms, float(total_pt), e2e_s, float(e2e_pt)], dtype=torch.float64, device=dev)
    if world == 1:
        return total_ms, float(total_pt), e2e_s, float(e2e_pt)
    mx = vals.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = vals.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx[0].item(), sm[1].item(), mx[2].item(), sm[3].item()


def run_ours(args):
    import torch
    import torch.distributed as dist

    lib = importlib.import_module(PKG + ".lib")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    eles, p, n, scale = workload(args.workload, rank)
    if args.particles:
        n = args.particles
    T = args.turns_per_step
    ctx = lib.Context(local)
    lat = lib.Lattice(ctx, eles, p)
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", local)
    vec0 = rings.matched_gaussian(eles, n, seed=rank, scale=scale)
    hb = lib.HostBunch.from_vec(vec0, p)

    def device_bunch():
        t = {k: torch.from_numpy(getattr(hb, k)).to(dev) for k in ("vec", "beta", "state", "ix_ele", "ix_turn", "location")}
        torch.cuda.synchronize()
        view = abi.Bunch(n, t["vec"].data_ptr(), t["beta"].data_ptr(), None, t["state"].data_ptr(),
                         t["ix_ele"].data_ptr(), t["ix_turn"].data_ptr(), t["location"].data_ptr())
        return t, view

    # launch shape: the library's autotuner (one-turn trials on a copy of the bunch)
    t, v = device_bunch()
    best = lib.autotune(ctx, lat, v)

    t, v = device_bunch()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    turn = 0
    # several ranks: each step's per-turn moment sums [T, 28] of the rank's shard, added over the
    # ranks by one all_reduce (the path's only exchange); timed with the kernel
    mom = torch.zeros((T, abi.N_MOMENTS), dtype=torch.float64, device=dev) if world > 1 else None
    job_moments = None

    def step(timed):
        nonlocal turn, job_moments
        alive0 = t["state"] == abi.ALIVE
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.check(lib.load().bmadgpu_track_bunch_device(ctx.handle, lat.handle, ctypes.byref(v), 0, lat.n_ele, turn, T,
                                                        mom.data_ptr() if mom is not None else None))
        if mom is not None:
            torch.cuda.current_stream().wait_stream(stream)
            job_moments = lib.allreduce_moments(mom)
            e1.record(torch.cuda.current_stream())
        else:
            e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        alive1 = t["state"] == abi.ALIVE
        lost_now = alive0 & ~alive1
        pt = int(alive1.sum().item()) * T + int((t["ix_turn"][lost_now] - turn + 1).sum().item())
        turn += T
        flush.fill_(1.0)
        torch.cuda.synchronize()
        return ms, pt

    for _ in range(args.warmup):
        step(False)
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launch_count
    total_ms, total_pt = 0.0, 0
    for _ in range(args.steps):
        ms, pt = step(True)
        total_ms += ms
        total_pt += pt
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = ctx.launch_count - launches0
    clk = clocks.stop()
    n_alive_end = int((t["state"] == abi.ALIVE).sum().item())

    # e2e: the public host-pointer API, copies included, on the bunch as it stands
    hb_e2e = lib.HostBunch(t["vec"].cpu().numpy(), t["beta"].cpu().numpy(), state=t["state"].cpu().numpy())
    pinned = {}
    for k in ("vec", "beta", "state", "ix_ele", "ix_turn", "location"):
        a = getattr(hb_e2e, k)
        pa = torch.from_numpy(a).pin_memory()
        pinned[k] = pa
        setattr(hb_e2e, k, pa.numpy())
    lib.track_bunch(ctx, lat, hb_e2e, n_turns=T, turn0=turn)   # warm the staging buffers
    if world > 1:
        dist.barrier()
    e2e_s, e2e_pt = 0.0, 0
    for _ in range(args.steps):
        alive0 = hb_e2e.state == abi.ALIVE
        t0 = time.perf_counter()
        lib.track_bunch(ctx, lat, hb_e2e, n_turns=T, turn0=turn)
        e2e_s += time.perf_counter() - t0
        alive1 = hb_e2e.state == abi.ALIVE
        lost_now = alive0 & ~alive1
        e2e_pt += int(alive1.sum()) * T + int((hb_e2e.ix_turn[lost_now] - turn + 1).sum())
        turn += T
    bytes_per = 6 * 8 + 8 + 4 * 4
    total_ms_max, total_pt_sum, e2e_s_max, e2e_pt_sum = combine_ranks(total_ms, total_pt, e2e_s, e2e_pt, world, dev)
    value = total_pt_sum / (total_ms_max / 1e3)
    e2e_value = e2e_pt_sum / e2e_s_max

    if rank == 0:
        ops, ops_split = op_count(eles, p, scale)
        peak = ctx.measure_fp64_peak()
        per_gpu = total_pt / (total_ms / 1e3)
        achieved = ops * per_gpu / 1e12
        traffic = None
        prof = os.path.join(ROOT, "profiles", "k_track_traffic.json")
        if os.path.exists(prof):
            try:
                tj = json.load(open(prof))
                if tj.get("workload") == args.workload:
                    traffic = tj["dram_bytes_per_particle_per_launch"] * n
            except (ValueError, KeyError):
                traffic = None
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded matched Gaussian bunch)",
            "config": dict(config_dict(args, n, lat.n_ele), tuning=best),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_per * n,
                    "d2h_bytes_per_step": bytes_per * n},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / (peak / 1e12), "traffic": traffic,
                         "ops_per_particle_turn": ops, "ops_split": ops_split,
                         "peak_source": "measured live: DFMA-chain probe on every SM (bmadgpu_measure_fp64_peak)"},
            "gpu_launches": launches,
            "clocks": clk,
            "particles_alive_end": n_alive_end,
        }
        if job_moments is not None:
            out["job_n_live_end"] = float(job_moments[-1, 0].item())
        if world == 1:
            out["cpu_baseline"] = cpu_baseline(eles, p, scale)
    lat.close()
    ctx.close()
    if rank == 0 and world == 1 and args.workload == "ring200" and not args.no_extras:
        # the benchmark's other headline figures, each from its own timed region on this GPU
        out.update(headline_extras(args, peak))
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_cr_ring(args, peak, steps=3, warmup=3):
    """ring200 with libbmadgpu_cr.so (correctly rounded transcendentals; bit-identical to the
    oracle run with a correctly rounded libm): device-resident particle-turns/s, L2 flushed between
    steps, the library's autotuned shape."""
    import torch
    lib = importlib.import_module(PKG + ".lib")
    previous = lib.get_math()
    lib.set_math("cr")
    try:
        eles, p, n, scale = workload("ring200", 0)
        T = args.turns_per_step
        ctx = lib.Context(0)
        lat = lib.Lattice(ctx, eles, p)
        dev = torch.device("cuda", 0)
        hb = lib.HostBunch.from_vec(rings.matched_gaussian(eles, n, seed=0, scale=scale), p)
        t = {k: torch.from_numpy(getattr(hb, k)).to(dev) for k in ("vec", "beta", "state", "ix_ele", "ix_turn", "location")}
        torch.cuda.synchronize()
        v = abi.Bunch(n, t["vec"].data_ptr(), t["beta"].data_ptr(), None, t["state"].data_ptr(),
                      t["ix_ele"].data_ptr(), t["ix_turn"].data_ptr(), t["location"].data_ptr())
        best = lib.autotune(ctx, lat, v)
        turn, tot_s, tot_pt = 0, 0.0, 0
        clocks = None
        for i in range(warmup + steps):
            if i == warmup:
                clocks = ClockSampler(0)
            state0 = t["state"].cpu().numpy()
            _flush_l2(dev)
            sec = _timed(ctx, lambda: lib.check(lib.load().bmadgpu_track_bunch_device(
                ctx.handle, lat.handle, ctypes.byref(v), 0, lat.n_ele, turn, T, None)))
            st, it = t["state"].cpu().numpy(), t["ix_turn"].cpu().numpy()
            pt = int((st == abi.ALIVE).sum()) * T + int((it[(state0 == abi.ALIVE) & (st != abi.ALIVE)] - turn + 1).sum())
            turn += T
            if i >= warmup:
                tot_s += sec
                tot_pt += pt
        clk = clocks.stop()
        value = tot_pt / tot_s
        ops, _ = op_count(eles, p, scale)
        out = {"value": value, "unit": UNIT, "steps": steps, "warmup": warmup, "ms_per_step": 1e3 * tot_s / steps,
               "library": "libbmadgpu_cr.so", "tuning": best, "clocks": clk,
               "workload": "ring200 as the main line (%d particles, %d turns per step)" % (n, T),
               "parity": "bit-identical to the oracle run with a correctly rounded libm (tests/test_gpu_bitexact.py)",
               "roofline": _fp64_roofline(ops * value, peak, "%.0f ops per particle-turn" % ops) if peak else None}
        lat.close()
        ctx.close()
        return out
    finally:
        lib.set_math(previous)


def headline_extras(args, peak):
    """Sub-records of the default line: the batched 256-variant job, a 200-job served stream and
    the adjoint gradient, each with its comparison against the plain kernel and its FP64 roofline."""
    ns = lambda **kw: argparse.Namespace(**dict(vars(args), **kw))
    b = run_batch(ns(steps=1, warmup=1, variants=256, plain_sample=8, turns_per_step=10), peak)
    sv = run_serve(ns(jobs=200, plain_sample=8), peak)
    ad = run_adjoint(ns(steps=3, warmup=1), peak)
    keep = lambda d, *ks: {k: d[k] for k in ks if k in d}
    cr = run_cr_ring(args, peak)
    return {
        "correctly_rounded": cr,
        "batched": dict(keep(b, "value", "unit", "ms_per_step", "e2e", "clocks", "gpu_launches"),
                        workload=b["config"]["workload"], tuning=b["config"]["tuning"],
                        vs_plain=b["plain_kernel"]["ratio"], plain_kernel=b["plain_kernel"],
                        roofline=b.get("roofline")),
        "served": dict(keep(sv, "value", "unit", "ms_per_step", "latency_s", "fma", "server", "clocks", "gpu_launches"),
                       workload=sv["config"]["workload"], vs_plain=sv["plain_kernel"]["ratio"],
                       plain_kernel=sv["plain_kernel"], roofline=sv.get("roofline")),
        "adjoint": dict(keep(ad, "value", "unit", "ms_per_step", "forward_equivalent", "fd_check", "clocks",
                             "gpu_launches"), workload=ad["config"]["workload"], roofline=ad.get("roofline")),
    }


def _timed(ctx, fn):
    """Device time of fn() on the context stream (CUDA events, synchronised both sides)."""
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    ctx.synchronize()
    return e0.elapsed_time(e1) / 1e3


def _particle_turns(state, ix_turn, turn0, n_turns):
    alive = state == abi.ALIVE
    lost = ~alive & (ix_turn >= turn0)
    return int(alive.sum()) * n_turns + int((ix_turn[lost] - turn0 + 1).sum())


def _flush_l2(dev):
    import torch
    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    buf.fill_(1.0)
    torch.cuda.synchronize()


def run_batch(args, peak=None):
    """256 lattice variants, dynamic-aperture grids, 2048 turns, batched path vs plain kernel.
    Returns the JSON line; peak (FP64 flop/s), if given, adds its roofline."""
    import torch
    lib = importlib.import_module(PKG + ".lib")
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n_var, n_turns = args.variants, 2048 if args.turns_per_step == 10 else args.turns_per_step
    rng = np.random.default_rng(2)
    counts = np.exp(rng.uniform(math.log(1024), math.log(65536), n_var)).astype(np.int64)
    ctx = lib.Context(0)
    lats, bunches = [], []
    for v in range(n_var):
        e, p = rings.perturbed_ring(50, seed=1000 + v)
        lats.append(lib.Lattice(ctx, e, p))
        bunches.append(lib.HostBunch.from_vec(rings.da_grid(int(counts[v])), p))
    whole = lib.concat_bunches(bunches)
    pinned = lib.PinnedBunch(whole.vec, whole.beta, state=whole.state, t=whole.t)
    batch = lib.Batch(ctx, lats, counts)
    batch.upload(-1, pinned)
    tuning = batch.autotune(sample_turns=32)
    out_b = lib.HostBunch(np.zeros((6, whole.n)), np.zeros(whole.n), t=np.zeros(whole.n))

    def one_step(timed):
        batch.upload(-1, pinned)
        ctx.synchronize()
        _flush_l2(dev)
        s = _timed(ctx, lambda: batch.track(n_turns))
        batch.download(-1, out_b)
        return s, _particle_turns(out_b.state, out_b.ix_turn, 0, n_turns)

    for _ in range(args.warmup):
        one_step(False)
    clocks = ClockSampler(0)
    l0 = ctx.launch_count
    tot_s, tot_pt = 0.0, 0
    for _ in range(args.steps):
        sec, pt = one_step(True)
        tot_s += sec
        tot_pt += pt
    launches = ctx.launch_count - l0
    clk = clocks.stop()
    value = tot_pt / tot_s
    # end to end: host arrays in, results out, every step, through the public API
    e2e_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        batch.upload(-1, pinned)
        batch.track(n_turns)
        batch.download(-1, out_b)
        e2e_s += time.perf_counter() - t0
    e2e = tot_pt / e2e_s
    # plain kernel, variant by variant, on a random sample (device-resident, its own autotuned
    # launch shape, the batch's compaction interval)
    sample = np.random.default_rng(5).choice(n_var, size=min(args.plain_sample, n_var), replace=False)
    big = int(np.argmax(counts))
    bt = {k: torch.from_numpy(np.array(getattr(bunches[big], k))).to(dev) for k in ("vec", "beta", "state")}
    plain_tuning = lib.autotune(ctx, lats[big], abi.Bunch(bunches[big].n, bt["vec"].data_ptr(), bt["beta"].data_ptr(),
                                                          None, bt["state"].data_ptr(), None, None, None))
    ctx.set_tuning(turns_per_launch=tuning["turns_per_launch"], compact=1)
    p_s, p_pt = 0.0, 0
    for v in sample:
        b = bunches[v]
        t = {k: torch.from_numpy(np.array(getattr(b, k))).to(dev) for k in ("vec", "beta", "state", "ix_ele", "ix_turn",
                                                                          "location")}
        view = abi.Bunch(b.n, t["vec"].data_ptr(), t["beta"].data_ptr(), None, t["state"].data_ptr(),
                         t["ix_ele"].data_ptr(), t["ix_turn"].data_ptr(), t["location"].data_ptr())
        _flush_l2(dev)
        sec = _timed(ctx, lambda: lib.check(lib.load().bmadgpu_track_bunch_device(
            ctx.handle, lats[v].handle, ctypes.byref(view), 0, lats[v].n_ele, 0, n_turns, None)))
        p_s += sec
        p_pt += _particle_turns(t["state"].cpu().numpy(), t["ix_turn"].cpu().numpy(), 0, n_turns)
    plain = p_pt / p_s
    out = {
        "metric": "particle-turns/s (FP64, batched 256-variant DA job)", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (perturbed rings, dynamic-aperture grids)",
        "config": {"workload": "batch256: %d perturbed 50-cell rings, %d particles (log-uniform 1024-65536 per "
                               "variant), %d turns from the initial grids per step" % (n_var, int(counts.sum()), n_turns),
                   "tuning": tuning, "l2": "flushed before each step (256 MiB write)"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(whole.n) * (8 * 8 + 4 * 4),
                "d2h_bytes_per_step": int(whole.n) * (8 * 8 + 4 * 4)},
        "plain_kernel": {"value": plain, "unit": UNIT, "ratio": value / plain,
                         "sample": "%d of %d variants, each tracked alone (device-resident, autotuned shape %s, "
                                   "compaction every %d turns), %.1f s" % (len(sample), n_var, plain_tuning,
                                                                          tuning["turns_per_launch"], p_s)},
        "gpu_launches": launches, "clocks": clk,
    }
    if peak:
        ops, _ = op_count(*rings.perturbed_ring(50, seed=1000), 1.0)
        out["roofline"] = _fp64_roofline(ops * value, peak, "%.0f ops per particle-turn (perturbed 50-cell ring)" % ops)
    batch.close()
    for lat in lats:
        lat.close()
    ctx.close()
    return out


def _fp64_roofline(ops_per_s, peak, what):
    return {"bound": "fp64", "achieved": ops_per_s / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
            "frac": ops_per_s / peak, "ops": what}


def run_serve(args, peak=None):
    """The Poisson stream of tracking jobs through the continuous-batching server. Returns the
    JSON line; peak (FP64 flop/s), if given, adds its roofline."""
    import threading
    import torch
    lib = importlib.import_module(PKG + ".lib")
    torch.cuda.set_device(0)
    ctx = lib.Context(0)
    stream = rings.serving_stream(args.jobs, seed=3)
    jobs = []
    t_prep = time.time()
    for j in stream:
        e, p = rings.perturbed_ring(j["cells"], seed=j["variant_seed"])
        lat = lib.Lattice(ctx, e, p)
        if j["kind"] == "gauss":
            vec = rings.matched_gaussian(e, j["n"], seed=j["variant_seed"] % 100000)
            j["fma"] = None
        else:
            # frequency-map job: grid offsets from the closed orbit, with the reference's set-up.
            # A perturbed ring whose closed orbit cannot be found (frequency_map itself would stop
            # there) is tracked as a plain grid job and counted.
            try:
                orbit, norm, tunes = lib.fma_setup(ctx, lat)
                vec = rings.fma_grid(j["n"]) + orbit[:, None]
                j["fma"] = (norm, orbit, tunes)
            except lib.BmadGpuError:
                vec = rings.fma_grid(j["n"])
                j["fma"] = None
                j["no_orbit"] = True
        hb = lib.HostBunch.from_vec(vec, p)
        jobs.append((j, lat, vec, hb.beta))
    t_prep = time.time() - t_prep
    n_fma = sum(1 for j, _, _, _ in jobs if j["fma"] is not None)
    n_no_orbit = sum(1 for j, _, _, _ in jobs if j.get("no_orbit"))

    def pinned_inputs():
        return [lib.PinnedBunch(vec, beta) for (_, _, vec, beta) in jobs]

    def server():
        # a quarter of HBM for resident particles, most of the rest for frequency-map records
        free_b = torch.cuda.mem_get_info(0)[0]
        return lib.Server(ctx, hbm_fraction=0.25, record_mib=int(0.6 * free_b / 2 ** 20))

    def submit(srv, j, lat, b, turns):
        if j["fma"] is None:
            return srv.submit(lat, b, turns)
        norm, orbit, tunes = j["fma"]
        return srv.submit_fma(lat, b, turns, norm, orbit, tunes)

    fma_summary = {}

    def run_stream(bunches):
        srv = server()
        start = time.perf_counter()
        ids = []
        for (j, lat, _, _), b in zip(jobs, bunches):
            dt = start + j["arrival"] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append((j, submit(srv, j, lat, b, j["turns"])))
        srv.wait(-1, timeout=7200)
        st = srv.stats()
        st["job_pt"] = [(j["cells"], srv.job(jid)["particle_turns"]) for j, jid in ids]
        done = [srv.fma_result(jid)[1] for j, jid in ids if j["fma"] is not None]
        fma_summary["particles_with_tunes"] = int(sum(int(np.sum(x == 0)) for x in done))
        fma_summary["particles"] = int(sum(len(x) for x in done))
        srv.close()
        return st

    # warm-up: a server with the first few jobs of the stream, shortened to 8 turns each
    warm = server()
    warm_b = [lib.PinnedBunch(vec, beta) for (_, _, vec, beta) in jobs[:3]]
    for (j, lat, _, _), b in zip(jobs[:3], warm_b):
        submit(warm, j, lat, b, 8)
    warm.wait(-1, timeout=600)
    warm.close()
    clocks = ClockSampler(0)
    l0 = ctx.launch_count
    st = run_stream(pinned_inputs())
    clk = clocks.stop()
    value = st["particle_turns"] / st["elapsed_s"]
    # plain kernel: jobs one after another (host buffers, synchronous), on a random sample, at the
    # plain kernel's default shape (the fastest measured on the 50- and 200-cell rings), compacting
    # the live list every 64 turns
    ctx.set_tuning(block=256, ctas_per_sm=2, stage_smem=1, turns_per_launch=64, compact=1)
    sample = np.random.default_rng(7).choice(len(jobs), size=min(args.plain_sample, len(jobs)), replace=False)
    p_s, p_pt = 0.0, 0
    for k in sample:
        j, lat, vec, beta = jobs[k]
        b = lib.HostBunch(vec, beta)
        t0 = time.perf_counter()
        lib.track_bunch(ctx, lat, b, n_turns=j["turns"])
        p_s += time.perf_counter() - t0
        p_pt += _particle_turns(b.state, b.ix_turn, 0, j["turns"])
    plain = p_pt / p_s
    n_part = sum(j["n"] for j, _, _, _ in jobs)
    out = {
        "metric": "particle-turns/s (FP64, served mixed request stream)", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * st["elapsed_s"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Poisson stream, perturbed rings, Gaussian / frequency-map grids)",
        "config": {"workload": "serve: first %d jobs of the 2000-job stream (mean gap 5 ms), %d particles, "
                               "50/100/200/400-cell rings, %d frequency-map jobs (turn-by-turn record and tunes on "
                               "the device; %d more whose ring has no closed orbit tracked as plain grids)"
                               % (len(jobs), n_part, n_fma, n_no_orbit),
                   "host_prep_s": t_prep},
        "fma": fma_summary,
        "latency_s": {"p50": st["latency_p50_s"], "p99": st["latency_p99_s"], "max": st["latency_max_s"]},
        "server": {k: st[k] for k in ("jobs_done", "rounds", "particle_turns", "capacity", "peak_resident",
                                      "gpu_busy_s", "gpu_idle_s", "gpu_max_gap_s")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": n_part * (8 * 8 + 4 * 4),
                "d2h_bytes_per_step": n_part * (8 * 8 + 4 * 4)},
        "plain_kernel": {"value": plain, "unit": UNIT, "ratio": value / plain,
                         "sample": "%d of %d jobs, one after another through bmadgpu_track_bunch (host buffers), "
                                   "%.1f s" % (len(sample), len(jobs), p_s)},
        "gpu_launches": ctx.launch_count - l0, "clocks": clk,
    }
    if peak:
        ops = {c: op_count(*rings.perturbed_ring(c, seed=7), 1.0)[0] for c in sorted({c for c, _ in st["job_pt"]})}
        work = sum(ops[c] * pt for c, pt in st["job_pt"])
        out["roofline"] = _fp64_roofline(work / st["elapsed_s"], peak, "per job: ops per particle-turn of its ring "
                                         "(%s) x its particle-turns" % ", ".join("%d cells %.0f" % kv for kv in ops.items()))
    for _, lat, _, _ in jobs:
        lat.close()
    ctx.close()
    return out


def run_adjoint(args, peak=None):
    """Gradient of the tracking loss with respect to 200 strengths by the adjoint kernel. Returns
    the JSON line; peak (FP64 flop/s), if given, adds its roofline, counting only the three
    forward passes of the sweep (tracking, segment and turn recomputation), not the adjoint's own
    operations."""
    import torch
    lib = importlib.import_module(PKG + ".lib")
    torch.cuda.set_device(0)
    ctx = lib.Context(0)
    eles, p = rings.ring(50)
    vec = rings.matched_gaussian(eles, 4096, seed=2)
    param_ele = [i for i, e in enumerate(eles) if e.key in (abi.QUADRUPOLE, abi.SEXTUPOLE)]
    lat = lib.Lattice(ctx, eles, p)
    b = lib.HostBunch.from_vec(vec, p)
    for _ in range(args.warmup):
        lib.loss_grad(ctx, lat, b, 256, param_ele, 16)
    clocks = ClockSampler(0)
    l0 = ctx.launch_count
    secs = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        loss, grad = lib.loss_grad(ctx, lat, b, 256, param_ele, 16)
        secs.append(time.perf_counter() - t0)
    clk = clocks.stop()
    fd_check = None
    gold = os.path.join(ROOT, "tests", "golden", "adjoint_config4_fd.json")
    if os.path.exists(gold):
        d = json.load(open(gold))
        fd_check = [{"slot": e["slot"], "attr": e["attr"], "h": e["h"], "fd": e["fd"], "adjoint": float(grad[e["slot"]]),
                     "rel_diff": abs(float(grad[e["slot"]]) - e["fd"]) / abs(e["fd"])} for e in d["entries"]]
    s = sum(secs) / len(secs)
    out = {
        "metric": "gradient evaluations/s (FP64 adjoint, 200 strengths)", "value": 1 / s, "unit": "gradients/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded matched Gaussian bunch)",
        "config": {"workload": "adjoint: 50-cell ring, 4096 particles, 256 turns, loss mean(x^2+y^2), "
                               "d/d(100 quad k1, 100 sextupole k2), checkpoints every 16 turns"},
        "forward_equivalent": {"value": 4096 * 256 / s, "unit": "particle-turns/s (forward part of the sweep)"},
        "e2e": {"value": 1 / s, "unit": "gradients/s", "h2d_bytes_per_step": 4096 * (8 * 8 + 4),
                "d2h_bytes_per_step": 8 * 201},
        "loss": loss, "fd_check": fd_check, "gpu_launches": ctx.launch_count - l0, "clocks": clk,
    }
    if peak:
        ops, _ = op_count(eles, p, 1.0)
        out["roofline"] = _fp64_roofline(3 * ops * 4096 * 256 / s, peak, "3 forward passes x %.0f ops per particle-"
                                         "turn (the adjoint's own operations not counted)" % ops)
    lat.close()
    ctx.close()
    return out


def run_kinds(args):
    """ns per particle-element of the plain kernel for each element kind of ring200."""
    import copy
    import torch
    lib = importlib.import_module(PKG + ".lib")
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx = lib.Context(0)
    n = args.particles or 1 << 20
    eles200, p = rings.ring(200, fringe=True, multipole_sigma=1e-4)
    plain, _ = rings.ring(200)
    nofringe, _ = rings.ring(200, fringe=False)
    cell = eles200[:9]
    kinds = {"drift": [cell[0], cell[2]], "quadrupole": [cell[1], cell[6]], "sbend": [nofringe[3]],
             "sbend_hwang_edges": [cell[3]], "sextupole": [plain[5], plain[7]],
             "sextupole_b3_b10": [cell[5], cell[7]], "ring200": None}
    # small amplitudes, so that few particles are lost in one pass through 1800 copies without
    # focusing; still far above the 1e-9 bounds of the exact bend's near-zero-orbit branch
    vec0 = rings.matched_gaussian(eles200, n, seed=1, scale=0.003)
    pc = p.p0c * (1 + vec0[5])
    beta0 = torch.from_numpy(pc / np.sqrt(pc * pc + p.mass * p.mass)).to(dev)
    out, alive_end = {}, {}
    clocks = ClockSampler(0)
    for name, proto in kinds.items():
        if proto is None:
            eles = eles200
        else:
            eles = [copy.deepcopy(proto[i % len(proto)]) for i in range(1800)]
            rings.set_ref_time(eles, p)
        lat = lib.Lattice(ctx, eles, p)
        init = {"vec": torch.from_numpy(np.ascontiguousarray(vec0)).to(dev), "beta": beta0,
                "state": torch.ones(n, dtype=torch.int32, device=dev)}
        t = {k: x.clone() for k, x in init.items()}
        v = abi.Bunch(n, t["vec"].data_ptr(), t["beta"].data_ptr(), None, t["state"].data_ptr(), None, None, None)
        run = lambda: lib.check(lib.load().bmadgpu_track_bunch_device(ctx.handle, lat.handle, ctypes.byref(v), 0,
                                                                      lat.n_ele, 0, 1, None))

        def reset():
            # every pass starts from the initial bunch: a lattice of one kind has no focusing, and
            # the sextupole kicks grow without bound over repeated passes
            for k in t:
                t[k].copy_(init[k])
            torch.cuda.synchronize()
        secs = []
        for i in range(args.warmup + args.steps):
            reset()
            _flush_l2(dev)
            sec = _timed(ctx, run)
            if i >= args.warmup:
                secs.append(sec)
        s_min = min(secs)
        out[name] = s_min / (n * len(eles)) * 1e9
        alive_end[name] = int((t["state"] == abi.ALIVE).sum())
    clk = clocks.stop()
    line = {
        "metric": "ns per particle-element (FP64 plain kernel, by element kind)", "value": out["ring200"],
        "unit": "ns/particle-element", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": False, "dtype": "f64", "data": "synthetic (seeded matched Gaussian, 0.003 sigma)",
        "config": {"workload": "kinds: 1800 copies of each element kind of ring200, %d particles, 1 turn per step, "
                               "best of the steps, L2 flushed between steps" % n, "tuning": ctx.get_tuning()},
        "kinds": out, "alive_end": alive_end, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    eles, p, n, scale = workload(args.workload, rank)
    threads = load_oracle().oracle_max_threads()
    sample_n, sample_t = (4096, 2) if args.workload == "ring200" else (4096, 20)
    vec = rings.matched_gaussian(eles, sample_n, seed=0, scale=scale)
    for _ in range(args.warmup):
        oracle_rate(eles, p, vec[:, :256], 1, threads)
    tot_pt, tot_s = 0.0, 0.0
    for _ in range(args.steps):
        rate, dt = oracle_rate(eles, p, vec, sample_t, threads)
        tot_pt += sample_n * sample_t
        tot_s += dt
    value = tot_pt / tot_s
    sample = "%d particles x %d turn(s) per step of the same ring, C++ oracle (restatement of the Fortran path), OpenMP %d threads" % (
        sample_n, sample_t, threads)
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded matched Gaussian bunch)", "config": config_dict(args, n, len(eles)),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["ring200", "ring50", "batch256", "serve", "adjoint", "kinds"],
                    default="ring200")
    ap.add_argument("--jobs", type=int, default=200, help="serve: number of jobs of the stream")
    ap.add_argument("--variants", type=int, default=256, help="batch256: number of lattice variants")
    ap.add_argument("--plain-sample", type=int, default=12, help="batch256/serve: variants/jobs timed on the plain path")
    ap.add_argument("--turns-per-step", type=int, default=10)
    ap.add_argument("--particles", type=int, default=0)
    ap.add_argument("--no-extras", action="store_true",
                    help="ring200: leave out the batched, served and adjoint sub-records of the default line")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("batch256", "serve", "adjoint"):
        import torch
        lib = importlib.import_module(PKG + ".lib")
        torch.cuda.set_device(0)
        c = lib.Context(0)
        peak = c.measure_fp64_peak()
        c.close()
        fn = {"batch256": run_batch, "serve": run_serve, "adjoint": run_adjoint}[args.workload]
        print(json.dumps(fn(args, peak)), flush=True)
    elif args.workload == "kinds":
        run_kinds(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
