"""The benchmark's larger mills on the device against the oracle, bit for bit: the DEM-only
configuration at 2,000, 20,000 and 200,000 discs (drum scaled to hold them) and the 5,000-disc
mill at fluid resolution 200 (~50.8k fluid particles), besides the 500-disc and resolution-100
cases of the golden fixtures (test_golden.py)."""
from __future__ import annotations

import time

import pytest

from milldynamics3_b200 import workloads as W
from milldynamics3_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _both(device, oracle, build, plan):
    out = []
    for b in (device, oracle):
        p, balls = build(b)
        s = Simulation(b, p, initial_balls=balls)
        t0 = time.perf_counter()
        for kind, count in plan:
            for _ in range(count):
                if kind == "frame":
                    s.step(1.0 / 60.0)
                else:
                    s.step_fixed()
        dt = time.perf_counter() - t0
        out.append((s.state_hash(True), s.counts(), s.last_step_stats()[2].to_dict(), dt))
        s.close()
    return out


@pytest.mark.parametrize("n_balls,plan", [(2000, [("frame", 2)]), (20000, [("frame", 1)]),
                                          (200000, [("sub", 1)])])
def test_dem_only_large_mills_match_the_oracle(device, oracle, n_balls, plan):
    (hd, cd, kd, td), (ho, co, ko, to) = _both(device, oracle, lambda b: W.dem_only(b, n_balls), plan)
    print("\nDEM-only %d discs: device %.3f s, oracle %.3f s, counters %s" % (n_balls, td, to, kd))
    assert cd == co == (n_balls, 0)
    assert kd == ko
    assert hd == ho


@pytest.mark.parametrize("viscosity", [1e-3, 1e-1])
def test_resolution_200_mill_matches_the_oracle(device, oracle, viscosity):
    (hd, cd, kd, td), (ho, co, ko, to) = _both(device, oracle, lambda b: W.large(b, 200, viscosity), [("sub", 2)])
    print("\nres-200 mill (mu %g): %s, device %.3f s, oracle %.3f s, counters %s" % (viscosity, cd, td, to, kd))
    assert cd == co and cd[1] > 50000
    assert kd == ko
    assert hd == ho
