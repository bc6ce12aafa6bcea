"""Seed sweeps on the device (all seeds one batch, one launch per frame) give, seed by seed,
exactly the oracle's run_seed results (batch.rs:40-107), dry and with slurry."""
from __future__ import annotations

import pytest

from milldynamics3_b200 import seeds
from milldynamics3_b200.sim import MillError, Simulation

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.seed == b.seed
    assert a.window_s == b.window_s
    assert a.coarse_graining_factor == b.coarse_graining_factor
    assert a.names == b.names
    assert a.values == b.values, [(n, x, y) for n, x, y in zip(a.names, a.values, b.values) if x != y]
    assert a.power_drift_rel_per_rev == b.power_drift_rel_per_rev


def test_stress_metrics_match_oracle(device, oracle):
    out = []
    for b in (device, oracle):
        p = b.preset(b.params_default(), "realtime")
        s = Simulation(b, p)
        for _ in range(3):
            s.step(1.0 / 60.0)
        out.append(s.stress_metrics().to_dict())
        s.close()
    assert out[0] == out[1]


def test_dry_sweep_matches_oracle_seed_by_seed(device, oracle):
    ss = [1, 2, 3, 11]
    pd = device.params_default()
    pd.slurry.enabled = 0
    po = oracle.params_default()
    po.slurry.enabled = 0
    dev = seeds.run_seeds(device, pd, ss, 1.0, 1.0)
    assert len(dev) == len(ss)
    for s, r in zip(ss, dev):
        _same(r, seeds.run_seed(oracle, po, s, 1.0, 1.0))
    assert abs(dev[0].window_s - 0.6) < 0.02
    assert dev[0].values != dev[1].values
    cd, co = seeds.combine(device, dev), seeds.combine(oracle, dev)
    assert cd.mean == co.mean and cd.std_err == co.std_err


def test_wet_sweep_matches_oracle_seed_by_seed(device, oracle):
    ss = [4, 5]
    pd = device.preset(device.params_default(), "realtime")
    po = oracle.preset(oracle.params_default(), "realtime")
    dev = seeds.run_seeds(device, pd, ss, 0.25, 1.0)
    for s, r in zip(ss, dev):
        _same(r, seeds.run_seed(oracle, po, s, 0.25, 1.0))


def test_sweep_rejects_what_the_oracle_rejects(device):
    p = device.params_default()
    with pytest.raises(MillError):
        seeds.run_seeds(device, p, [1], 1.0, 0.5)
    with pytest.raises(MillError):
        seeds.run_seeds(device, p, [], 1.0, 1.0)
