"""The drag and buoyancy sweeps give the same bits whichever order their warps take balls in
(MgOptions.sweep_order: by dependency level, the default, or by ball index), with any number of
sweep warps, and the oracle's bits."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200 import workloads
from milldynamics3_b200.sim import MillError, Simulation

pytestmark = pytest.mark.gpu


def _run(backend, p, frames, balls=None, **opts):
    s = Simulation(backend, p, balls) if balls is not None else Simulation(backend, p)
    if opts:
        s.set_options(**opts)
    for _ in range(frames):
        s.step(1.0 / 60.0)
    out = (s.state_hash(True), s.scalars().to_dict(), s.stress_histogram_rate(), s.last_step_stats()[2].to_dict())
    s.close()
    return out


@pytest.mark.parametrize("workload", ["realtime", "realtime_300"])
def test_sweep_order_does_not_change_results(device, oracle, workload):
    p, balls = getattr(workloads, workload)(device)
    ref = _run(device, p, 3, balls, sweep_order=1)
    for opts in (dict(sweep_order=0), dict(sweep_order=0, sweep_warps=4), dict(sweep_order=0, mill_blocks=1),
                 dict(sweep_order=1, sweep_warps=7)):
        got = _run(device, p, 3, balls, **opts)
        assert got[0] == ref[0], opts
        assert got[1] == ref[1] and got[3] == ref[3], opts
        assert np.array_equal(got[2], ref[2]), opts
    po, bo = getattr(workloads, workload)(oracle)
    assert _run(oracle, po, 3, bo)[0] == ref[0]


def test_sweep_order_bounds(device):
    s = Simulation(device, device.preset(device.params_default(), "realtime"))
    with pytest.raises(MillError):
        s.set_options(sweep_order=2)
    s.set_options(sweep_order=1)
    s.close()
