"""Benchmark of the mill sub-step path on one B200 (one process per GPU).

Workload (default): the 'realtime' preset mill exactly as Params supplies it (63 mm drum, 407
ZrO2 discs of 2 mm, water slurry at resolution 25, 24 sub-steps per 1/60 s frame), stepped frame
by frame through the library. One "step" is one frame (24 coupled sub-steps).

  value   sub-steps/s with the mill state resident in device memory (Simulation::step calls).
  e2e     the same through the C ABI with host buffers: each step uploads the state from pinned
          host memory, steps the frame and reads the state back (the drop-in for a caller that
          owns the state on the host, as coupling::step_recorded's callers do).

--impl reference times the oracle (the C++ restatement of the reference's Rust sub-step; the
reference toolchain is not available) on the host cores, on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sub-steps/s (1 mill) & batched mill-frames/s on 1 B200; p50/p99 frame latency"
UNIT = "sub-steps/s"
# DRAM bytes (read + write) of one realtime frame launch, from an ncu capture (see profiles/)
REALTIME_LAUNCH_DRAM_BYTES = 2.076e6 + 0.273e6


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def bytes_model(tot, n_sub, nf, nb, dem_iters):
    """Algorithmic bytes of the sub-steps summed in `tot` (the per-pass stream model: each array
    read or written once per pass, neighbour gathers not counted as extra traffic)."""
    (density_it, cg_it, groups, links, _in_range, pairs, edges, _active, items, _r) = tot
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
    path = os.path.join(ROOT, "gpurun_out", "bench_clocks.csv")
    os.makedirs(os.path.dirname(path), exist_ok=True)
    try:
        f = open(path, "w")
        p = subprocess.Popen(["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                              "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                             stdout=f, stderr=subprocess.DEVNULL)
        return p, f, path
    except Exception:
        return None, None, path


def clocks_stop(h, gpu_index=0):
    p, f, path = h
    if p is None:
        return None
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    f.close()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
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


def make_sim(backend, preset="realtime"):
    from milldynamics3_b200.sim import Simulation
    p = backend.preset(backend.params_default(), preset)
    return Simulation(backend, p), p


def run_reference(args):
    """The oracle (C++ restatement of the reference's single-threaded Rust sub-step) on host cores."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import ORACLE_EXTRA, build_oracle
    from milldynamics3_b200 import capi
    from milldynamics3_b200.sim import Backend
    b = Backend(capi.Lib(build_oracle(), "or_", ORACLE_EXTRA))
    sim, p = make_sim(b)
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
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "realtime preset, 1 mill (63 mm drum, %d discs, %d fluid particles, "
                                   "%d sub-steps/frame)" % (nb, nf, n_sub), "step": "one 1/60 s frame"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": "%d frames of the realtime mill, single thread" % args.steps},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(seconds=10.0):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import ORACLE_EXTRA, build_oracle
    from milldynamics3_b200 import capi
    from milldynamics3_b200.sim import Backend
    b = Backend(capi.Lib(build_oracle(), "or_", ORACLE_EXTRA))
    sim, p = make_sim(b)
    n_sub = b.derived(p).effective_substeps
    sim.step(1.0 / 60.0)
    frames = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        sim.step(1.0 / 60.0)
        frames += 1
    dt = time.perf_counter() - t0
    # metrics::compute on the same state, one thread
    calls = 0
    t1 = time.perf_counter()
    while calls < 5 or time.perf_counter() - t1 < 1.0:
        sim.metrics()
        calls += 1
    met_ms = 1e3 * (time.perf_counter() - t1) / calls
    # surface::extract_surface on the same state, one thread
    calls = 0
    t1 = time.perf_counter()
    while calls < 5 or time.perf_counter() - t1 < 1.0:
        sim.surface_flat()
        calls += 1
    surf_ms = 1e3 * (time.perf_counter() - t1) / calls
    return {"value": frames * n_sub / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "%d frames of the realtime mill on the oracle (C++ restatement), 1 thread, %.1f s"
                      % (frames, dt), "metrics_ms_per_call": met_ms, "surface_ms_per_call": surf_ms}


def run_batched(lib, backend, args):
    """The 512-mill mix in one launch per frame (mg_batch_*), against the plain path (each mill
    stepped alone, one after another) sampled on the same mix. Returns the 'batched' object."""
    import numpy as np
    import torch
    from milldynamics3_b200.batch import Batch, mix_params
    from milldynamics3_b200.sim import Simulation
    ps, info = mix_params(backend, args.batch_mills, seed=1)
    d = [backend.derived(p) for p in ps]
    batch = Batch(backend, ps)
    foot = C.c_uint64()
    total_bytes = 0
    for i in range(len(ps)):
        lib.sim_footprint(batch.mill(i).h, C.byref(foot))
        total_bytes += foot.value
    stream = torch.cuda.ExternalStream(batch.stream())
    for _ in range(max(args.warmup, 3)):
        batch.step_frames(1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.batch_frames):
        t0 = time.perf_counter()
        batch.step_frames(1)
        lat.append(time.perf_counter() - t0)
    ev1.record(stream)
    torch.cuda.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    kernel_ms, _ = batch.last_kernel_ms()
    batch.close()
    mfps = args.batch_frames * len(ps) / t
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
    lat_ms = sorted(1e3 * x for x in lat)
    return {"mills": len(ps), "mill_frames_per_s": mfps, "ms_per_batch_frame": 1e3 * t / args.batch_frames,
            "kernel_ms_per_batch_frame": kernel_ms, "frames_timed": args.batch_frames,
            "frame_latency_ms": {"p50": lat_ms[len(lat_ms) // 2], "max": lat_ms[-1]},
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


def run_serving(backend, args, plain_mfps):
    """The request server under a Poisson stream of jobs drawn from the 512-mill mix's
    distribution (mean args.serve_rate requests/s, horizons uniform in 0.5-10 s simulated, a
    150 GiB admission budget), for args.serve_seconds of wall time. Every step admits what has
    arrived and fits, advances all running jobs by one frame in one launch and retires finished
    jobs. Frame latency: the wall time from the start of the step that computes a job's frame to
    its end (what a client waiting for that frame sees)."""
    import numpy as np
    from milldynamics3_b200 import capi
    from milldynamics3_b200.batch import mix_params
    from milldynamics3_b200.server import Server
    pool, _ = mix_params(backend, 1024, seed=3)
    rng = np.random.default_rng(7)
    server = Server(backend, memory_budget_bytes=150 << 30, max_active=args.serve_max_active)
    lat, waits, active = [], [], []
    submitted = finished = frames = 0
    t_start = time.perf_counter()
    next_arrival = t_start + rng.exponential(1.0 / args.serve_rate)
    while time.perf_counter() - t_start < args.serve_seconds:
        now = time.perf_counter()
        while next_arrival <= now:
            server.submit(pool[submitted % len(pool)], float(rng.uniform(0.5, 10.0)))
            submitted += 1
            next_arrival += rng.exponential(1.0 / args.serve_rate)
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
        lat.extend([1e3 * dt] * n_adv)
        active.append(n_adv)
    elapsed = time.perf_counter() - t_start
    st = server.stats()
    server.close()
    lat.sort()
    waits.sort()
    pct = lambda a, q: a[min(len(a) - 1, int(q * len(a)))] if a else None
    mfps = frames / elapsed
    return {"requests_per_s": args.serve_rate, "seconds": elapsed, "submitted": submitted, "finished": finished,
            "still_queued": st.queued, "mill_frames": frames, "mill_frames_per_s": mfps,
            "frame_latency_ms": {"p50": pct(lat, 0.5), "p99": pct(lat, 0.99)},
            "admission_wait_s": {"p50": pct(waits, 0.5), "p99": pct(waits, 0.99)},
            "running_jobs_mean": float(sum(active) / max(len(active), 1)), "max_active": args.serve_max_active,
            "plain_mill_frames_per_s": plain_mfps,
            "ratio_vs_plain": mfps / plain_mfps if plain_mfps else None,
            "workload": "Poisson arrivals of mills drawn from the 512-mill mix distribution, horizons U[0.5,10] s "
                        "simulated, 150 GiB admission budget, one launch per frame for all running jobs"}


def run_device(args):
    import numpy as np
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from milldynamics3_b200 import capi, native
    from milldynamics3_b200.sim import Backend
    lib = native.load()
    b = Backend(lib)
    sim, p = make_sim(b)
    d = b.derived(p)
    n_sub = d.effective_substeps
    nb, nf = sim.counts()
    stream_ptr = C.c_void_p()
    lib.sim_stream(sim.h, C.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    for _ in range(max(args.warmup, 3)):
        sim.step(1.0 / 60.0)
    lib.counter_totals(sim.h, None, None, 1)
    # ---- value: state resident on the device
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    ck = clocks_start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        sim.step(1.0 / 60.0)
        ms = C.c_float()
        lib.sim_last_kernel_ms(sim.h, C.byref(ms), None)
        kernel_ms.append(ms.value)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clocks_stop(ck, local)
    t = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        tt = torch.tensor([t], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    value = world * args.steps * n_sub / t
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
    launches = C.c_uint64()
    lib.sim_last_kernel_ms(sim.h, None, C.byref(launches))
    # metrics::compute through the C ABI (one kernel launch, result copied back), per call
    sim.metrics()
    t0 = time.perf_counter()
    for _ in range(20):
        sim.metrics()
    met_ms = 1e3 * (time.perf_counter() - t0) / 20
    # Simulation::fluid_surface through the C ABI (two kernel launches, flattened polygons copied
    # back into a host buffer), per call
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
                "config": {"workload": "realtime preset, 1 mill per GPU (63 mm drum, %d discs, %d fluid "
                                       "particles, %d sub-steps/frame)" % (nb, nf, n_sub),
                           "step": "one 1/60 s frame", "l2": "working set (~%.1f MB) is L2-resident; no flush "
                           "between steps (successive frames read the state the last one wrote)"
                           % (per_launch_bytes / n_sub / 1e6),
                           "ms_per_frame": 1e3 * t / args.steps, "parallelism": "replicas" if world > 1 else "1 mill"},
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
        plain_mfps = None
        if args.batch_mills > 0:
            line["batched"] = run_batched(lib, b, args)
            plain_mfps = line["batched"]["plain_mill_frames_per_s"]
        if args.serve_seconds > 0:
            line["serving"] = run_serving(b, args, plain_mfps)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
            line["metrics"]["cpu_ms_per_call"] = line["cpu_baseline"].pop("metrics_ms_per_call")
            line["surface"]["cpu_ms_per_call"] = line["cpu_baseline"].pop("surface_ms_per_call")
        print(json.dumps(line), flush=True)
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
    ap.add_argument("--batch-mills", type=int, default=512, help="mills of the batched leg (0: skip it)")
    ap.add_argument("--batch-frames", type=int, default=5)
    ap.add_argument("--plain-sample", type=int, default=16, help="mills of the mix timed on the plain path")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="wall seconds of the serving leg (0: skip it)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="mean job arrivals per second")
    ap.add_argument("--serve-max-active", type=int, default=1024, help="jobs advanced per launch at most")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_device(args)


if __name__ == "__main__":
    main()
