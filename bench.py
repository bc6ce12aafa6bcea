"""Benchmark of the mill sub-step path on one B200 (one process per GPU).

Workload (the headline line): the 'realtime' preset mill exactly as Params supplies it (63 mm
drum, 407 ZrO2 discs of 2 mm, water slurry at resolution 25, 24 sub-steps per 1/60 s frame),
stepped frame by frame through the library. One "step" is one frame (24 coupled sub-steps).

  value   sub-steps/s with the mill state resident in device memory (Simulation::step calls).
  e2e     the same through the C ABI with host buffers: each step uploads the state from pinned
          host memory, steps the frame and reads the state back (the drop-in for a caller that
          owns the state on the host, as coupling::step_recorded's callers do).

Further legs in the same line (rank 0): the other configurations (300 random steel discs; DEM-only
2,000 and 20,000 discs; the 5,000-disc mill at fluid resolution 100 and 200), each beside the CPU
oracle's time on a bounded sample; the batched 512-mill mix (throughput, p50/p99 frame latency,
HBM roofline, the host's share, a CPU baseline of one oracle process per host core); the request
server under an overloaded, a sustainable and a memory-bound Poisson load.

--impl reference times the oracle (the C++ restatement of the reference's Rust sub-step; the
reference toolchain is not available) on the host cores, on the headline workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sub-steps/s (1 mill) & batched mill-frames/s on 1 B200; p50/p99 frame latency"
UNIT = "sub-steps/s"
# DRAM bytes (read + write) of one realtime frame launch, from an ncu capture (see profiles/)
REALTIME_LAUNCH_DRAM_BYTES = 2.435e6 + 0.377e6
# The headline workload's description, the same in both arms' lines.
CONFIG = {"workload": "realtime preset, 1 mill per GPU (63 mm drum, 407 ZrO2 discs of 2 mm, 794 fluid particles at "
                      "resolution 25, 24 sub-steps per 1/60 s frame)",
          "step": "one 1/60 s frame (24 coupled sub-steps)",
          "l2": "the mill's working set (~3 MB) is L2-resident; no flush between steps (each frame reads the state "
                "the last one wrote)",
          "parallelism": "1 mill per GPU (replicas across GPUs)"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def bytes_model(tot, n_sub, nf, nb, dem_iters):
    """Algorithmic bytes of the sub-steps summed in `tot` (the per-pass stream model: each array
    read or written once per pass, neighbour gathers not counted as extra traffic)."""
    (density_it, cg_it, groups, links, _in_range, pairs, edges, _active, items, _ccd) = tot
    N, B, K = float(nf), float(nb), float(dem_iters)
    s = float(n_sub)
    cells = N  # dense fluid grid: about one cell per particle at cell size h
    per_sub = (40 * N + 24 * N + 8 * cells + 12 * N + 32 * N + 24 * B + 20 * N + 16 * N + 20 * B + 56 * N
               + 48 * B + 16 * N + 12 * N + 20 * N + 56 * N + B * 200)
    total = s * per_sub
    total += 4 * edges * (1 + 1 + 1 + 1)  # CSR build, cohesion, recompute, shear: 4E each
    total += density_it * 44 * N + 8 * edges * (density_it / max(s, 1.0))
    total += 48 * items + 24 * groups + 24 * links
    total += cg_it * (120 * N + 24 * groups / max(s, 1.0) + 64 * B) + 16 * edges * (cg_it / max(s, 1.0))
    total += pairs * (8 + 40 * K + 120)
    return total


def clocks_start():
    """nvidia-smi clock and throttle samples every 200 ms into a temporary file."""
    f = tempfile.NamedTemporaryFile("w", prefix="bench_clocks_", suffix=".csv", delete=False)
    try:
        p = subprocess.Popen(["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                              "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
        return p, f, f.name
    except Exception:
        return None, f, f.name


def clocks_stop(h, gpu_index=0):
    p, f, path = h
    if p is not None:
        p.terminate()
        try:
            p.wait(timeout=5)
        except Exception:
            p.kill()
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        lines = open(path).read().splitlines()
        os.unlink(path)
    except OSError:
        lines = []
    for line in lines:
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9 or parts[0] != str(gpu_index):
            continue
        try:
            sm.append(float(parts[1]))
            mx = float(parts[2])
        except ValueError:
            continue
        for nm, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    if not sm:
        return None
    sm.sort()
    return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def pct(a, q):
    a = sorted(a)
    return a[min(len(a) - 1, int(q * len(a)))] if a else None


def oracle_backend(build=True):
    """The oracle (test infrastructure: only the CPU-baseline leg and the reference arm use it);
    built first unless `build` is false (the baseline's worker processes load what the parent
    built)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import ORACLE_EXTRA, ORACLE_SO, build_oracle
    from milldynamics3_b200 import capi
    from milldynamics3_b200.sim import Backend
    return Backend(capi.Lib(build_oracle() if build else ORACLE_SO, "or_", ORACLE_EXTRA))


def run_reference(args):
    """The oracle (C++ restatement of the reference's single-threaded Rust sub-step) on host cores."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from milldynamics3_b200 import workloads
    from milldynamics3_b200.sim import Simulation
    b = oracle_backend()
    p, _ = workloads.realtime(b)
    sim = Simulation(b, p)
    n_sub = b.derived(p).effective_substeps
    for _ in range(args.warmup):
        sim.step(1.0 / 60.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.step(1.0 / 60.0)
    dt = time.perf_counter() - t0
    v = args.steps * n_sub / dt
    nb, nf = sim.counts()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (Params + seed)", "config": dict(CONFIG),
            "particle_updates_per_s": v * (nb + nf),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": "%d frames of the realtime mill on the oracle (C++ restatement of the "
                                       "reference's Rust sub-step), single thread" % args.steps},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _oracle_substeps_per_s(b, build, seconds, max_substeps=None):
    from milldynamics3_b200.sim import Simulation
    p, balls = build(b)
    s = Simulation(b, p, initial_balls=balls)
    s.step_fixed()
    n = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds and (max_substeps is None or n < max_substeps):
        s.step_fixed()
        n += 1
    dt = time.perf_counter() - t0
    s.close()
    return n / dt, n, dt


def cpu_baseline(seconds, config_legs):
    """The oracle on the box's host: the realtime mill on one thread (~`seconds`), metrics and the
    free surface per call, and a bounded sample of each further configuration."""
    from milldynamics3_b200 import workloads
    from milldynamics3_b200.sim import Simulation
    b = oracle_backend()
    p, _ = workloads.realtime(b)
    sim = Simulation(b, p)
    n_sub = b.derived(p).effective_substeps
    sim.step(1.0 / 60.0)
    frames = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        sim.step(1.0 / 60.0)
        frames += 1
    dt = time.perf_counter() - t0
    calls = 0
    t1 = time.perf_counter()
    while calls < 5 or time.perf_counter() - t1 < 1.0:
        sim.metrics()
        calls += 1
    met_ms = 1e3 * (time.perf_counter() - t1) / calls
    calls = 0
    t1 = time.perf_counter()
    while calls < 5 or time.perf_counter() - t1 < 1.0:
        sim.surface_flat()
        calls += 1
    surf_ms = 1e3 * (time.perf_counter() - t1) / calls
    legs = {}
    for name, (build, _frames) in config_legs.items():
        v, n, t = _oracle_substeps_per_s(b, build, 2.0, max_substeps=2000)
        legs[name] = {"sub_steps_per_s": v, "sample": "%d sub-steps, %.2f s, 1 thread" % (n, t)}
    return {"value": frames * n_sub / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "%d frames of the realtime mill on the oracle (C++ restatement), 1 thread, %.1f s"
                      % (frames, dt), "metrics_ms_per_call": met_ms, "surface_ms_per_call": surf_ms,
            "configs": legs}


def config_legs():
    """The further configurations of the bench line: name -> (builder(backend), frames timed)."""
    from milldynamics3_b200 import workloads as W
    return {
        "1b_realtime_300_steel_discs": (W.realtime_300, 10),
        "2_dem_only_2000_discs": (lambda b: W.dem_only(b, 2000), 20),
        "2_dem_only_20000_discs": (lambda b: W.dem_only(b, 20000), 3),
        "3_5000_discs_res100": (lambda b: W.large(b, 100, 1e-3), 3),
        "3_5000_discs_res200": (lambda b: W.large(b, 200, 1e-3), 2),
    }


def run_configs(lib, backend, legs):
    """Each further configuration on the device: sub-steps/s over a few frames after one warm-up
    frame (CUDA events on the handle's stream)."""
    import torch
    from milldynamics3_b200.sim import Simulation
    out = {}
    for name, (build, frames) in legs.items():
        p, balls = build(backend)
        s = Simulation(backend, p, initial_balls=balls)
        n_sub = backend.derived(p).effective_substeps
        nb, nf = s.counts()
        sp = C.c_void_p()
        lib.sim_stream(s.h, C.byref(sp))
        stream = torch.cuda.ExternalStream(sp.value)
        s.step(1.0 / 60.0)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(frames):
            s.step(1.0 / 60.0)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3
        v = frames * n_sub / t
        out[name] = {"balls": nb, "fluid": nf, "sub_steps_per_frame": n_sub, "frames_timed": frames,
                     "sub_steps_per_s": v, "ms_per_frame": 1e3 * t / frames, "particle_updates_per_s": v * (nb + nf)}
        s.close()
    return out


def _oracle_mill_frames(job):
    """One host process of the config-4 CPU baseline: one frame of each of its mills on the
    oracle (Params as bytes); returns (mill-frames, seconds)."""
    pbytes_list, frames = job
    from milldynamics3_b200 import capi
    from milldynamics3_b200.sim import Simulation
    b = oracle_backend(build=False)
    sims = [Simulation(b, capi.Params.from_buffer_copy(pb)) for pb in pbytes_list]
    t0 = time.perf_counter()
    for _ in range(frames):
        for s in sims:
            s.step(1.0 / 60.0)
    dt = time.perf_counter() - t0
    for s in sims:
        s.close()
    return len(sims) * frames, dt


def batched_cpu_baseline(ps, pool, per_proc=4):
    """Config 4 on the host: one oracle process per core, each stepping `per_proc` mills of the
    mix one frame (a bounded sample); aggregate mill-frames/s."""
    import numpy as np
    n = os.cpu_count() or 1
    rng = np.random.default_rng(5)
    pick = rng.choice(len(ps), size=min(len(ps), n * per_proc), replace=False)
    jobs = [([bytes(ps[i]) for i in pick[k::n]], 1) for k in range(n)]
    t0 = time.perf_counter()
    res = pool.map(_oracle_mill_frames, jobs)
    wall = time.perf_counter() - t0
    mf = sum(r[0] for r in res)
    # every process's own stepping time (their loads do not overlap perfectly with pool start-up)
    slowest = max(r[1] for r in res)
    return {"mill_frames_per_s": mf / slowest, "processes": n, "mill_frames": mf, "seconds": slowest,
            "wall_s_including_start": wall, "kind": "port",
            "sample": "%d mills of the mix, one frame each, one oracle process per host core" % mf}


def run_batched(lib, backend, args, pool):
    """The 512-mill mix in one launch per frame (mg_batch_*), against the plain path (each mill
    stepped alone, one after another) sampled on the same mix. Returns the 'batched' object."""
    import numpy as np
    import torch
    from milldynamics3_b200 import capi
    from milldynamics3_b200.batch import Batch, mix_params
    from milldynamics3_b200.sim import Simulation
    from milldynamics3_b200.autotune import Autotuner
    ps, info = mix_params(backend, args.batch_mills, seed=1)
    d = [backend.derived(p) for p in ps]
    # the block shape: the autotuner's pick on this mix (every candidate's mill states compared),
    # unless given on the command line
    tuned = None
    if args.batch_threads or args.batch_regs:
        opts = {"block_threads": args.batch_threads, "block_regs": args.batch_regs}
    else:
        tuned = Autotuner(backend, frames=2).tune_batch(ps)
        opts = tuned.options
    batch = Batch(backend, ps)
    batch.set_options(**opts)
    foot = C.c_uint64()
    total_bytes = 0
    mills = [batch.mill(i) for i in range(len(ps))]
    for m in mills:
        lib.sim_footprint(m.h, C.byref(foot))
        total_bytes += foot.value
    stream = torch.cuda.ExternalStream(batch.stream())
    for _ in range(max(args.warmup, 3)):
        batch.step_frames(1)
    for m in mills:
        lib.counter_totals(m.h, None, None, 1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat, kms = [], []
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.batch_frames):
        t0 = time.perf_counter()
        batch.step_frames(1)
        lat.append(time.perf_counter() - t0)
        kms.append(batch.last_kernel_ms()[0])
    ev1.record(stream)
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    # algorithmic bytes of the timed frames, mill by mill (counters counted on the device)
    alg = 0.0
    tot = (C.c_uint64 * 10)()
    nsum = C.c_uint64()
    for i, m in enumerate(mills):
        lib.counter_totals(m.h, tot, C.byref(nsum), 0)
        nb, nf = m.counts()
        alg += bytes_model(list(tot), nsum.value, nf, nb, ps[i].simulation.dem_iterations)
    batch.close()
    mfps = args.batch_frames * len(ps) / t
    k_ms = sum(kms) / len(kms)
    hbm, peak_kind = peaks()
    achieved = alg / args.batch_frames / (k_ms / 1e3) / 1e9
    # plain path on a sample of the same mix: each mill alone, one frame after one warm-up frame
    rng = np.random.default_rng(2)
    sample = sorted(rng.choice(len(ps), size=min(args.plain_sample, len(ps)), replace=False).tolist())
    plain_t = []
    for i in sample:
        s = Simulation(backend, ps[i])
        s.step(1.0 / 60.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.step(1.0 / 60.0)
        torch.cuda.synchronize()
        plain_t.append(time.perf_counter() - t0)
        s.close()
    plain_mfps = 1.0 / (sum(plain_t) / len(plain_t))
    nb = np.array([x.eff_ball_count for x in d])
    ns = np.array([x.effective_substeps for x in d])
    res = np.array([x.effective_fluid_resolution for x in d])
    lat_ms = [1e3 * x for x in lat]
    out = {"mills": len(ps), "mill_frames_per_s": mfps, "ms_per_batch_frame": 1e3 * t / args.batch_frames,
           "kernel_ms_per_batch_frame": k_ms,
           "host_share": max(0.0, 1.0 - k_ms / (1e3 * t / args.batch_frames)), "frames_timed": args.batch_frames,
           "frame_latency_ms": {"p50": pct(lat_ms, 0.5), "p99": pct(lat_ms, 0.99), "max": max(lat_ms)},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                        "peak_kind": peak_kind, "kernel": "mill_substeps_kernel (one launch per batch frame)",
                        "algorithmic_bytes_per_launch": alg / args.batch_frames, "kernel_ms_per_launch": k_ms},
           "block_shape": opts, "autotune": None if tuned is None else {"picked": tuned.options,
                                                                        "ms_per_frame": tuned.timings},
           "plain_mill_frames_per_s": plain_mfps, "plain_sample_mills": len(sample),
           "ratio_vs_plain": mfps / plain_mfps, "device_bytes": total_bytes,
           "mix": {"balls_min_mean_max": [int(nb.min()), float(nb.mean()), int(nb.max())],
                   "substeps_min_mean_max": [int(ns.min()), float(ns.mean()), int(ns.max())],
                   "resolution_min_mean_max": [int(res.min()), float(res.mean()), int(res.max())],
                   "diameter_mm_min_max": [1e3 * min(x["diameter_m"] for x in info),
                                           1e3 * max(x["diameter_m"] for x in info)],
                   "sampling": "ball count log-uniform 100-3000 and fill U[0.2,0.4] with D = 2r sqrt(N/(J phi)) "
                               "redrawn until D in [40,120] mm; resolution U[15,60]; speed U[50,90]% critical; "
                               "2 mm discs; seed per mill"}}
    if pool is not None:
        out["cpu_baseline"] = batched_cpu_baseline(ps, pool)
        out["cpu_baseline"]["ratio"] = mfps / out["cpu_baseline"]["mill_frames_per_s"]
    return out


def serve(backend, rate, seconds, max_active, budget, pool_params, seed):
    """The request server under Poisson arrivals (mean `rate` jobs/s) of mills drawn from the mix,
    horizons uniform in 0.5-10 s simulated, for `seconds` of wall time. Every step admits what has
    arrived and fits, advances all running jobs by one frame in one launch and retires finished
    jobs. Frame latency: the wall time of the step that computes a job's frame."""
    import numpy as np
    from milldynamics3_b200 import capi
    from milldynamics3_b200.server import Server
    rng = np.random.default_rng(seed)
    server = Server(backend, memory_budget_bytes=budget, max_active=max_active)
    lat, waits, active, steps = [], [], [], []
    submitted = finished = frames = 0
    horizon_frames = 0.0
    t_start = time.perf_counter()
    next_arrival = t_start + rng.exponential(1.0 / rate)
    peak_bytes = 0
    while time.perf_counter() - t_start < seconds:
        now = time.perf_counter()
        while next_arrival <= now:
            h = float(rng.uniform(0.5, 10.0))
            server.submit(pool_params[submitted % len(pool_params)], h)
            horizon_frames += math.ceil(h * 60.0)
            submitted += 1
            next_arrival += rng.exponential(1.0 / rate)
        t0 = time.perf_counter()
        server.step()
        dt = time.perf_counter() - t0
        n_adv = 0
        for u in server.poll():
            if u.state in (capi.JOB_RUNNING, capi.JOB_FINISHED):
                n_adv += 1
                if u.frames_done == 1:
                    waits.append(u.queued_s)
            finished += u.state == capi.JOB_FINISHED
        frames += n_adv
        if n_adv:
            lat.extend([1e3 * dt] * n_adv)
            steps.append(1e3 * dt)
        active.append(n_adv)
        peak_bytes = max(peak_bytes, server.stats().device_bytes_in_use)
    elapsed = time.perf_counter() - t_start
    st = server.stats()
    server.close()
    return {"requests_per_s": rate, "seconds": elapsed, "submitted": submitted, "finished": finished,
            "still_queued": st.queued, "mill_frames": frames, "mill_frames_per_s": frames / elapsed,
            "offered_mill_frames_per_s": horizon_frames / elapsed,
            "frame_latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99)},
            "step_ms": {"p50": pct(steps, 0.5), "p99": pct(steps, 0.99)},
            "admission_wait_s": {"p50": pct(waits, 0.5), "p99": pct(waits, 0.99)},
            "running_jobs_mean": float(sum(active) / max(len(active), 1)), "running_jobs_max": max(active or [0]),
            "max_active": max_active, "memory_budget_bytes": budget, "peak_device_bytes_in_use": peak_bytes}


def run_serving(backend, args, capacity_mfps, plain_mfps):
    """Three loads of the request server: the north-star rate (200 jobs/s, far beyond capacity:
    the queue grows; labelled overloaded), a sustainable rate (offered mill-frames/s at 70 % of
    the measured batched capacity) and a memory-bound one (the 150 GiB footprint budget binds, not
    the active-job cap)."""
    from milldynamics3_b200.batch import mix_params
    pool, _ = mix_params(backend, 1024, seed=3)
    mean_frames = 60.0 * 5.25  # horizons U[0.5, 10] s
    out = {"workload": "Poisson arrivals of mills drawn from the 512-mill mix distribution, horizons U[0.5,10] s "
                       "simulated, one launch per frame for all running jobs",
           "plain_mill_frames_per_s": plain_mfps}
    runs = [("overloaded", args.serve_rate, args.serve_seconds, args.serve_max_active, 150 << 30)]
    if capacity_mfps:
        # twice the window: jobs live 5.25 s on average, so the population needs that long to settle
        runs.append(("sustainable", 0.7 * capacity_mfps / mean_frames, 2 * args.serve_seconds,
                     args.serve_max_active, 150 << 30))
    runs.append(("memory_bound", args.serve_rate * 10, args.serve_seconds, 1 << 20, 150 << 30))
    for k, (name, rate, secs, mx, budget) in enumerate(runs):
        r = serve(backend, rate, secs, mx, budget, pool, seed=7 + k)
        r["load"] = name
        r["ratio_vs_plain"] = r["mill_frames_per_s"] / plain_mfps if plain_mfps else None
        out[name] = r
    return out


def run_device(args):
    import numpy as np
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    # the config-4 CPU baseline's processes start before the first GPU call (spawn)
    pool = None
    if rank == 0 and not args.no_cpu_baseline and args.batch_mills > 0:
        import multiprocessing as mp
        oracle_backend()  # built once here; the workers only load it
        pool = mp.get_context("spawn").Pool(os.cpu_count() or 1)
    from milldynamics3_b200 import capi, native, workloads
    from milldynamics3_b200.sim import Backend, Simulation
    lib = native.load()
    b = Backend(lib)
    p, _ = workloads.realtime(b)
    sim = Simulation(b, p)
    d = b.derived(p)
    n_sub = d.effective_substeps
    nb, nf = sim.counts()
    stream_ptr = C.c_void_p()
    lib.sim_stream(sim.h, C.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    for _ in range(max(args.warmup, 3)):
        sim.step(1.0 / 60.0)
    # ---- value: state resident on the device; nothing but the frames inside the event pair
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck = clocks_start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step(1.0 / 60.0)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clocks_stop(ck, local)
    t = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        tt = torch.tensor([t], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    value = world * args.steps * n_sub / t
    # ---- the kernel's own launch time and the device counters, over the same number of frames
    lib.counter_totals(sim.h, None, None, 1)
    lib.stage_cycles(sim.h, None, 1)
    kernel_ms = []
    for _ in range(args.steps):
        sim.step(1.0 / 60.0)
        ms = C.c_float()
        lib.sim_last_kernel_ms(sim.h, C.byref(ms), None)
        kernel_ms.append(ms.value)
    tot = (C.c_uint64 * 10)()
    nsum = C.c_uint64()
    lib.counter_totals(sim.h, tot, C.byref(nsum), 0)
    per_launch_bytes = bytes_model(list(tot), nsum.value, nf, nb, p.simulation.dem_iterations) / max(args.steps, 1)
    cyc = (C.c_uint64 * 40)()
    lib.stage_cycles(sim.h, cyc, 1)
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    stages = {capi.STAGE_NAMES[q]: round(cyc[q] / max(nsum.value, 1) / mhz, 2) for q in range(40) if cyc[q]}
    k_ms = sum(kernel_ms) / len(kernel_ms)
    hbm, peak_kind = peaks()
    achieved = per_launch_bytes / (k_ms / 1e3) / 1e9
    # ---- e2e: host buffers through the C ABI, copies inside the timed region
    bl, fl = sim.balls(), sim.fluid()
    hb = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in bl.items()}
    hf = {k: torch.from_numpy(np.ascontiguousarray(fl[k])).pin_memory() for k in ("x", "v", "dye")}
    h2d = sum(t_.numel() * 4 for t_ in hb.values()) + sum(t_.numel() * 4 for t_ in hf.values())

    def fptr(t_):
        return C.cast(t_.data_ptr(), capi.f32p)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.set_balls(sim.h, nb, fptr(hb["x"]), fptr(hb["v"]), fptr(hb["theta"]), fptr(hb["omega"]))
        lib.set_fluid(sim.h, nf, fptr(hf["x"]), fptr(hf["v"]), fptr(hf["dye"]), None)
        sim.step(1.0 / 60.0)
        lib.get_balls(sim.h, fptr(hb["x"]), fptr(hb["v"]), fptr(hb["theta"]), fptr(hb["omega"]))
        lib.get_fluid(sim.h, fptr(hf["x"]), fptr(hf["v"]), fptr(hf["dye"]), None, None)
    torch.cuda.synchronize()
    te = time.perf_counter() - t0
    e2e = world * args.steps * n_sub / te
    # metrics::compute and Simulation::fluid_surface through the C ABI, per call
    sim.metrics()
    t0 = time.perf_counter()
    for _ in range(20):
        sim.metrics()
    met_ms = 1e3 * (time.perf_counter() - t0) / 20
    surf_buf = torch.zeros(capi.SURFACE_OUT_CAP, dtype=torch.float32).pin_memory()
    surf_len = C.c_uint32()
    lib.fluid_surface(sim.h, fptr(surf_buf), surf_buf.numel(), C.byref(surf_len))
    t0 = time.perf_counter()
    for _ in range(20):
        lib.fluid_surface(sim.h, fptr(surf_buf), surf_buf.numel(), C.byref(surf_len))
    surf_ms = 1e3 * (time.perf_counter() - t0) / 20
    surf_polys = int(surf_buf[0].item())
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (Params + seed)",
                "config": dict(CONFIG), "particle_updates_per_s": value * (nb + nf),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": REALTIME_LAUNCH_DRAM_BYTES, "peak_kind": peak_kind,
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one realtime "
                                               "frame launch (profiles/mill_substeps_kernel_realtime.md)",
                             "kernel": "mill_substeps_kernel (one launch per frame)",
                             "kernel_ms_per_launch": k_ms, "algorithmic_bytes_per_launch": per_launch_bytes},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
                "gpu_launches": args.steps, "clocks": clocks, "stage_us_per_substep": stages,
                "metrics": {"call": "mg_metrics (metrics::compute on the realtime mill's state, one kernel)",
                            "ms_per_call": met_ms},
                "surface": {"call": "mg_fluid_surface (surface::extract_surface on the realtime mill's state, "
                                    "two kernels, flattened polygons to a host buffer)",
                            "ms_per_call": surf_ms, "polygons": surf_polys, "floats": surf_len.value},
                "counters_per_substep": {f: round(tot[q] / max(nsum.value, 1), 2) for q, (f, _) in
                                         enumerate(capi.StepCounters._fields_)}}
        legs = config_legs()
        if not args.no_configs:
            line["configs"] = run_configs(lib, b, legs)
        plain_mfps = capacity = None
        if args.batch_mills > 0:
            line["batched"] = run_batched(lib, b, args, pool)
            plain_mfps = line["batched"]["plain_mill_frames_per_s"]
            capacity = line["batched"]["mill_frames_per_s"]
        if args.serve_seconds > 0:
            line["serving"] = run_serving(b, args, capacity, plain_mfps)
        if not args.no_cpu_baseline:
            cb = cpu_baseline(args.cpu_seconds, legs if not args.no_configs else {})
            line["metrics"]["cpu_ms_per_call"] = cb.pop("metrics_ms_per_call")
            line["surface"]["cpu_ms_per_call"] = cb.pop("surface_ms_per_call")
            for name, leg in cb.pop("configs").items():
                if name in line.get("configs", {}):
                    line["configs"][name]["cpu_baseline"] = leg
                    line["configs"][name]["ratio_vs_cpu"] = (line["configs"][name]["sub_steps_per_s"]
                                                             / leg["sub_steps_per_s"])
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if pool is not None:
        pool.close()
    sim.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="device", choices=["device", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the further configurations")
    ap.add_argument("--batch-mills", type=int, default=512, help="mills of the batched leg (0: skip it)")
    ap.add_argument("--batch-frames", type=int, default=50)
    ap.add_argument("--batch-threads", type=int, default=0, help="threads per mill block (0: the library's default)")
    ap.add_argument("--batch-regs", type=int, default=0, help="64: the 64-register build (two 512-thread blocks per SM)")
    ap.add_argument("--plain-sample", type=int, default=16, help="mills of the mix timed on the plain path")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="wall seconds of each serving run (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="mean job arrivals per second (overloaded run)")
    ap.add_argument("--serve-max-active", type=int, default=1024, help="jobs advanced per launch at most")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_device(args)


if __name__ == "__main__":
    main()
