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

    def step(timed):
        nonlocal turn
        alive0 = t["state"] == abi.ALIVE
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.check(lib.load().bmadgpu_track_bunch_device(ctx.handle, lat.handle, ctypes.byref(v), 0, lat.n_ele, turn, T, None))
        e1.record(stream)
        ctx.synchronize()
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
    vals = torch.tensor([total_ms, float(total_pt), e2e_s, float(e2e_pt)], dtype=torch.float64, device=dev)
    if world > 1:
        mx = vals.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = vals.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        total_ms_max, total_pt_sum, e2e_s_max, e2e_pt_sum = mx[0].item(), sm[1].item(), mx[2].item(), sm[3].item()
    else:
        total_ms_max, total_pt_sum, e2e_s_max, e2e_pt_sum = total_ms, float(total_pt), e2e_s, float(e2e_pt)
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
        if world == 1:
            out["cpu_baseline"] = cpu_baseline(eles, p, scale)
        print(json.dumps(out), flush=True)
    lat.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


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
    ap.add_argument("--workload", choices=["ring200", "ring50"], default="ring200")
    ap.add_argument("--turns-per-step", type=int, default=10)
    ap.add_argument("--particles", type=int, default=0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
