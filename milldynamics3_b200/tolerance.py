"""The A/B tolerance gate for physical metrics: the reference's `tolerance_probe`
(crates/mill-core/examples/tolerance_probe.rs), over this library.

Record a baseline, change the solver, then compare:

    python -m milldynamics3_b200.tolerance --baseline base.csv
    python -m milldynamics3_b200.tolerance --compare base.csv

The configurations, seeds (1..=N), window (settle, then measure, in drum revolutions), per-seed
window means, mean +- standard error over seeds and the gate rules are the reference's
(tolerance_probe.rs:11-27, 57-115, 181-193, 258-328, 330-344, 412-446), and the CSV layout is
the same (`config,metric,mean,se`, Rust `{:e}` numbers), so a baseline recorded by either tool
can be compared by the other. The difference is how the runs are scheduled: on the device
library every (config, seed) run whose frame counts agree is a mill of one batch, so a frame of
all of them is one launch; each mill's numbers are those of the same run alone. ms_per_frame
(informational in the reference) is then the batch's wall time per frame, shared by its mills.
"""
from __future__ import annotations

import argparse
import ctypes as C
import decimal
import math
import sys
import time
from dataclasses import dataclass

import numpy as np

from . import capi
from .sim import Backend, Simulation

F = np.float32
FPS = 60.0
SAMPLE_EVERY_FRAMES = 6   # tolerance_probe.rs:42


@dataclass(frozen=True)
class ProbeConfig:
    """tolerance_probe.rs:44-55"""
    name: str
    max_balls: int
    resolution: int
    shipped: bool
    viscosity_pa_s: float | None


# tolerance_probe.rs:57-115 (the same table: names and parameters are the interface of the
# baseline CSV files)
CONFIGS = (
    ProbeConfig("ui_fast", 300, 25, False, None),
    ProbeConfig("ui_accuracy", 600, 50, False, None),
    ProbeConfig("ship_fast", 300, 25, True, None),
    ProbeConfig("ship_acc", 600, 50, True, None),
    ProbeConfig("ship_v0.01", 300, 25, True, 0.01),
    ProbeConfig("ship_v1", 300, 25, True, 1.0),
    ProbeConfig("ship_v50", 300, 25, True, 50.0),
    ProbeConfig("ship_acc_v50", 600, 50, True, 50.0),
)

REL, ANGLE, ENERGY_FRACTION, COMPRESSION, INFO = "rel", "angle", "energy_fraction", "compression", "info"

# tolerance_probe.rs:181-193: metric names in report order, with their gate
METRICS = (
    ("power_w", REL),
    ("torque_nm", REL),
    ("specific_power_w_per_kg", REL),
    ("impacts_per_ball_per_s", REL),
    ("toe_angle_deg", ANGLE),
    ("shoulder_angle_deg", ANGLE),
    ("unattributed_over_shaft", ENERGY_FRACTION),
    ("compression_mean", COMPRESSION),
    ("compression_worst5pct", COMPRESSION),
    ("mean_shear_rate_per_s", INFO),
    ("ms_per_frame", INFO),
)


def gate_of(name: str) -> str:
    return dict(METRICS).get(name, INFO)


def _rem_euclid(x: float, m: float) -> float:
    r = math.fmod(x, m)
    return r + abs(m) if r < 0.0 else r


def circular_mean_deg(x) -> float:
    """Wrap-safe circular mean in degrees [0, 360); NaN if empty (tolerance_probe.rs:202-211)."""
    if len(x) == 0:
        return math.nan
    s = c = 0.0
    for d in x:
        s += math.sin(math.radians(d))
        c += math.cos(math.radians(d))
    return _rem_euclid(math.degrees(math.atan2(s, c)), 360.0)


def mean_or_nan(x) -> float:
    """tolerance_probe.rs:213-219 (sequential sum)"""
    if len(x) == 0:
        return math.nan
    s = 0.0
    for v in x:
        s += v
    return s / len(x)


def mean_se(v):
    """Mean and standard error (n - 1) of the finite values; NaN if none (tolerance_probe.rs:330-344)."""
    v = [a for a in v if math.isfinite(a)]
    if not v:
        return math.nan, math.nan
    n = float(len(v))
    m = 0.0
    for a in v:
        m += a
    m /= n
    if len(v) > 1:
        ss = 0.0
        for a in v:
            ss += (a - m) ** 2
        se = math.sqrt((ss / (n - 1.0)) / n)
    else:
        se = 0.0
    return m, se


def judge(gate: str, a, b):
    """(delta, pass) of a new (mean, se) b against a baseline a; pass is None for informational
    metrics (tolerance_probe.rs:412-446)."""
    am, ase = a
    bm, bse = b
    if gate == ANGLE and math.isfinite(am) and math.isfinite(bm):
        d = _rem_euclid(bm - am, 360.0)
        delta = d - 360.0 if d > 180.0 else d
    else:
        delta = bm - am
    if math.isnan(am) or math.isnan(bm):
        both = math.isnan(am) and math.isnan(bm)
        return (0.0 if both else math.nan), (None if gate == INFO else both)
    stat = 2.0 * math.sqrt(ase * ase + bse * bse)
    if gate == REL:
        return delta, abs(delta) <= max(stat, 0.02 * abs(am))
    if gate == ANGLE:
        return delta, abs(delta) <= max(stat, 2.0)
    if gate == ENERGY_FRACTION:
        return delta, abs(bm) <= abs(am) * 1.10 + 0.005
    if gate == COMPRESSION:
        return delta, bm <= am * 1.10 + 1e-4
    return delta, None


def params_for(backend: Backend, cfg: ProbeConfig, seed: int) -> capi.Params:
    """tolerance_probe.rs:222-256"""
    p = backend.params_default()
    if not cfg.shipped:
        p.mill.diameter_m = 1.0
        p.mill.speed_mode = capi.SPEED_PERCENT_CRITICAL
        p.mill.speed_value = 70.0
        p.mill.direction = capi.DIR_CCW
    p.lifters.count = 0
    p.slurry.enabled = 1
    if cfg.viscosity_pa_s is not None:
        p.slurry.viscosity_pa_s = cfg.viscosity_pa_s
    if not cfg.shipped:
        p.simulation.coarse_graining_mode = capi.CG_AUTO
    p.simulation.max_balls = cfg.max_balls
    p.simulation.resolution = cfg.resolution
    p.simulation.seed = seed
    backend.validate(p)
    return p


def to_vertical_degrees(atan2_rad: float, omega: float) -> float:
    """metrics.rs:275-279 in f32 (f32::to_degrees multiplies by 180/pi rounded to f32)."""
    sign = F(-1.0) if F(omega) >= 0.0 else F(1.0)
    v = F(sign * F(F(atan2_rad) - F(math.pi / 2)))
    deg = F(v * F(180.0 / math.pi))
    r = F(np.fmod(deg, F(360.0)))
    return float(F(r + F(360.0)) if r < 0.0 else r)


def window_frames(backend: Backend, p: capi.Params, settle_revs: float, measure_revs: float):
    """(settle, measure) frame counts of run_one (tolerance_probe.rs:265-267), f32 arithmetic."""
    rpm = F(backend.derived(p).rpm)
    rev_s = F(F(60.0) / rpm)

    def frames(revs):
        x = float(F(F(F(revs) * rev_s) * F(FPS)))
        r = math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)   # f32::round
        return max(int(r), 0)
    return frames(settle_revs), max(frames(measure_revs), 1)


def _div(a: float, b: float) -> float:
    """IEEE f64 division (inf or NaN for a zero divisor, as in Rust)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return float(np.float64(a) / np.float64(b))


class _Run:
    """One (config, seed) run's accumulators (tolerance_probe.rs:259-328)."""

    def __init__(self, cfg, seed, sim, omega):
        self.cfg, self.seed, self.sim, self.omega = cfg, seed, sim, omega
        self.impacts, self.toe, self.shoulder, self.comp_mean, self.comp_worst = [], [], [], [], []
        self.shear_sum = 0.0
        self.spec_e0 = 0.0

    def sample(self):
        s = self.sim
        stress = s.stress_metrics()
        self.impacts.append(float(stress.impacts_total_per_ball_per_s))
        m = s.metrics()
        if m.valid & capi.METRIC_TOE_SHOULDER:
            self.toe.append(to_vertical_degrees(m.toe_angle_rad, self.omega))
            self.shoulder.append(to_vertical_degrees(m.shoulder_angle_rad, self.omega))
        nf = s.counts()[1]
        rho0 = F(s.fluid_material().rest_density)
        if nf > 0 and rho0 > 0.0:
            r = s.fluid_densities().astype(F)
            c = np.fmax(F(r / rho0) - F(1.0), F(0.0)).astype(np.float64)
            self.comp_mean.append(float(np.cumsum(c)[-1]) / len(c))
            top = np.sort(c)[::-1][:max(len(c) // 20, 1)]
            self.comp_worst.append(float(np.cumsum(top)[-1]) / len(top))

    def result(self, measure_frames, ms_per_frame):
        s = self.sim
        eb = s.energy_budget()
        el = max(eb.elapsed_s, 1e-12)
        power = eb.shaft_work_j / el
        spec_e1 = float(s.stress_metrics().cumulative_specific_energy_j_per_kg)
        return [
            ("power_w", power),
            ("torque_nm", power / max(abs(float(self.omega)), 1e-12)),
            ("specific_power_w_per_kg", (spec_e1 - self.spec_e0) / el),
            ("impacts_per_ball_per_s", mean_or_nan(self.impacts)),
            ("toe_angle_deg", circular_mean_deg(self.toe)),
            ("shoulder_angle_deg", circular_mean_deg(self.shoulder)),
            ("unattributed_over_shaft", _div(eb.unattributed_j, eb.shaft_work_j)),
            ("compression_mean", mean_or_nan(self.comp_mean)),
            ("compression_worst5pct", mean_or_nan(self.comp_worst)),
            ("mean_shear_rate_per_s", self.shear_sum / measure_frames),
            ("ms_per_frame", ms_per_frame),
        ]


def run_group(backend: Backend, runs, settle_frames: int, measure_frames: int, batched: bool):
    """Steps the (config, seed) runs of one frame window side by side: as one batch (a launch per
    frame) when `batched`, else one Simulation after the other each frame. Returns, per run, its
    list of (metric, value)."""
    params = [params_for(backend, cfg, seed) for cfg, seed in runs]
    omegas = [float(backend.derived(p).omega) for p in params]
    if batched:
        from .batch import Batch
        batch = Batch(backend, params)
        sims = [batch.mill(i) for i in range(len(params))]

        def step():
            batch.step_frames(1, 1.0 / FPS)

        def shear():
            return [float(sc.mean_shear_rate_per_s) for sc in batch.scalars()]
    else:
        batch = None
        sims = [Simulation(backend, p) for p in params]

        def step():
            for sm in sims:
                sm.step(1.0 / FPS)

        def shear():
            return [float(sm.scalars().mean_shear_rate_per_s) for sm in sims]
    acc = [_Run(cfg, seed, sm, om) for (cfg, seed), sm, om in zip(runs, sims, omegas)]
    for _ in range(settle_frames):
        step()
    for a in acc:
        a.sim.reset_energy_budget()
        a.spec_e0 = float(a.sim.stress_metrics().cumulative_specific_energy_j_per_kg)
    step_s = 0.0
    for f in range(measure_frames):
        t = time.perf_counter()
        step()
        step_s += time.perf_counter() - t
        for a, g in zip(acc, shear()):
            a.shear_sum += g
        if f % SAMPLE_EVERY_FRAMES == 0:
            for a in acc:
                a.sample()
    ms = step_s * 1e3 / measure_frames
    out = [a.result(measure_frames, ms) for a in acc]
    if batch is not None:
        batch.close()
    else:
        for sm in sims:
            sm.close()
    return out


def run_all(backend: Backend, seeds: int = 3, settle_revs: float = 2.0, measure_revs: float = 3.0,
            only=None, batched: bool | None = None, log=None):
    """tolerance_probe.rs:348-376: {(config, metric): (mean, se)} over seeds 1..=seeds."""
    if batched is None:
        batched = hasattr(backend.lib, "batch_create")
    cfgs = [c for c in CONFIGS if only is None or c.name in only]
    groups = {}
    for cfg in cfgs:
        for s in range(seeds):
            p = params_for(backend, cfg, 1 + s)
            groups.setdefault(window_frames(backend, p, settle_revs, measure_revs), []).append((cfg, 1 + s))
    per = {}
    for (settle, measure), runs in groups.items():
        t = time.perf_counter()
        results = run_group(backend, runs, settle, measure, batched)
        if log:
            log("[%s] %d runs of %d + %d frames done in %.0fs" % (
                ",".join(sorted({c.name for c, _ in runs})), len(runs), settle, measure, time.perf_counter() - t))
        for (cfg, seed), r in zip(runs, results):
            for name, v in r:
                per.setdefault((cfg.name, name), []).append((seed, v))
    table = {}
    for key, vals in per.items():
        table[key] = mean_se([v for _, v in sorted(vals)])
    return table


def rust_exp(x: float) -> str:
    """Rust's `{:e}` of an f64: shortest round-trip digits, `d.ddde<exp>`."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0e0" if math.copysign(1.0, x) < 0 else "0e0"
    sign, digits, exp = decimal.Decimal(repr(x)).as_tuple()
    digits = "".join(map(str, digits)).rstrip("0") or "0"
    e = exp + len(decimal.Decimal(repr(x)).as_tuple().digits) - 1
    mant = digits[0] + ("." + digits[1:] if len(digits) > 1 else "")
    return ("-" if sign else "") + mant + "e" + str(e)


def write_csv(path: str, table) -> None:
    """tolerance_probe.rs:378-388"""
    out = ["config,metric,mean,se"]
    for cfg in CONFIGS:
        for name, _ in METRICS:
            if (cfg.name, name) in table:
                m, se = table[(cfg.name, name)]
                out.append("%s,%s,%s,%s" % (cfg.name, name, rust_exp(m), rust_exp(se)))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_csv(path: str):
    """tolerance_probe.rs:390-405"""
    table = {}
    with open(path) as f:
        lines = f.read().splitlines()[1:]
    for line in lines:
        if not line.strip():
            continue
        p = line.split(",")
        if len(p) != 4:
            raise ValueError(f"bad CSV line: {line}")
        table[(p[0], p[1])] = (float(p[2]), float(p[3]))
    return table


def compare(base, table, out=print):
    """The --compare report (tolerance_probe.rs:466-507); returns the number of failed gates."""
    failed = 0
    out("%-12s %-26s %13s %13s %10s  verdict" % ("config", "metric", "baseline", "new", "delta %"))
    for cfg in CONFIGS:
        if not any(k[0] == cfg.name for k in table):
            continue
        for name, _ in METRICS:
            key = (cfg.name, name)
            if key not in base or key not in table:
                out("%-12s %-26s missing in baseline or new run" % (cfg.name, name))
                continue
            a, b = base[key], table[key]
            delta, ok = judge(gate_of(name), a, b)
            pct = delta / abs(a[0]) * 100.0 if abs(a[0]) > 1e-300 else math.nan
            verdict = "info" if ok is None else ("PASS" if ok else "FAIL")
            failed += ok is False
            out("%-12s %-26s %13.6e %13.6e %+10.3f  %s" % (cfg.name, name, a[0], b[0], pct, verdict))
    return failed


def main(argv=None, backend=None) -> int:
    """The tolerance_probe command line on the device library, or on `backend` when one is given."""
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--seeds", type=int, default=3)
    ap.add_argument("--settle-revs", type=float, default=2.0)
    ap.add_argument("--measure-revs", type=float, default=3.0)
    ap.add_argument("--baseline")
    ap.add_argument("--compare")
    ap.add_argument("--only", type=lambda s: s.split(","))
    a = ap.parse_args(argv)
    if backend is None:
        from . import native
        backend = Backend(native.load())
    t0 = time.perf_counter()
    print("tolerance_probe: seeds=%d settle_revs=%g measure_revs=%g" % (a.seeds, a.settle_revs, a.measure_revs))
    table = run_all(backend, a.seeds, a.settle_revs, a.measure_revs, a.only,
                    log=lambda m: print(m, file=sys.stderr))
    print()
    print("%-12s %-26s %14s %12s" % ("config", "metric", "mean", "se"))
    for cfg in CONFIGS:
        for name, _ in METRICS:
            if (cfg.name, name) in table:
                m, se = table[(cfg.name, name)]
                print("%-12s %-26s %14.6e %12.3e" % (cfg.name, name, m, se))
    if a.baseline:
        write_csv(a.baseline, table)
        print("\nbaseline written to " + a.baseline)
    failed = 0
    if a.compare:
        print("\nCOMPARE against " + a.compare)
        failed = compare(read_csv(a.compare), table)
        print("\n%d gated metric(s) FAILED" % failed)
    print("total wall time: %.0fs" % (time.perf_counter() - t0))
    return 1 if failed else 0


if __name__ == "__main__":
    sys.exit(main())
