"""metrics::compute on the device (one kernel launch) gives exactly the oracle's fields."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _both(device, oracle, build, frames, balls=None):
    out = []
    for b in (device, oracle):
        s = Simulation(b, build(b), initial_balls=balls)
        for _ in range(frames):
            s.step(1.0 / 60.0)
        out.append((s.metrics().to_dict(), s.state_hash(True)))
        s.close()
    return out


def _realtime(b):
    return b.preset(b.params_default(), "realtime")


def _lifters(b):
    p = b.params_default()
    p.lifters.count = 8
    p.lifters.height_m = 0.004
    p.lifters.base_width_m = 0.006
    p.lifters.top_width_m = 0.003
    b.validate(p)
    return p


def _dry(b):
    p = b.params_default()
    p.slurry.enabled = 0
    return p


@pytest.mark.parametrize("build,frames", [(_realtime, 6), (_lifters, 4), (_dry, 3)])
def test_device_metrics_match_oracle(device, oracle, build, frames):
    (dm, dh), (om, oh) = _both(device, oracle, build, frames)
    assert dh == oh
    assert dm == om, {k: (dm[k], om[k]) for k in dm if dm[k] != om[k]}
    assert dm["valid"] & capi.METRIC_CENTROID


def test_device_metrics_of_empty_populations(device, oracle):
    (dm, _), (om, _) = _both(device, oracle, _dry, 0, balls=np.zeros((0, 2), np.float32))
    assert dm == om
    assert dm["valid"] == 0


def test_metrics_match_mixing_index_and_repeat(device):
    s = Simulation(device, _realtime(device))
    for _ in range(3):
        s.step(1.0 / 60.0)
    a, b = s.metrics().to_dict(), s.metrics().to_dict()
    assert a == b
    mi = s.mixing_index()
    assert (mi is None) == (not a["valid"] & capi.METRIC_MIXING)
    if mi is not None:
        assert a["mixing_index"] == mi
    s.close()


@pytest.mark.parametrize("frames", [0, 5])
def test_device_fluid_densities_match_oracle(device, oracle, frames):
    out = []
    for b in (device, oracle):
        s = Simulation(b, _realtime(b))
        for _ in range(frames):
            s.step(1.0 / 60.0)
        out.append(s.fluid_densities())
        s.close()
    assert len(out[0]) == len(out[1]) > 0
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))


def test_device_metrics_json_matches_oracle(device, oracle):
    from milldynamics3_b200 import wire
    out = []
    for b in (device, oracle):
        s = Simulation(b, _realtime(b))
        for _ in range(4):
            s.step(1.0 / 60.0)
        out.append(wire.metrics_to_json(s))
        s.close()
    assert out[0] == out[1]
