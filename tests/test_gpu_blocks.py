"""A single mill's per-ball stages spread over helper thread blocks (MgOptions.mill_blocks) give
exactly the results of the mill's block alone, and the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200.sim import MillError, Simulation

pytestmark = pytest.mark.gpu


def _run(backend, preset, frames, **opts):
    p = backend.preset(backend.params_default(), preset)
    s = Simulation(backend, p)
    if opts:
        s.set_options(**opts)
    for _ in range(frames):
        s.step(1.0 / 60.0)
    out = (s.state_hash(True), s.scalars().to_dict(), s.stress_histogram_rate(), s.last_step_stats()[2].to_dict())
    s.close()
    return out


@pytest.mark.parametrize("preset", ["realtime", "balanced"])
def test_mill_blocks_do_not_change_results(device, oracle, preset):
    ref = _run(device, preset, 2, mill_blocks=1)
    for mb in (2, 8, 16):
        got = _run(device, preset, 2, mill_blocks=mb)
        assert got[0] == ref[0], f"mill_blocks={mb}"
        assert got[1] == ref[1] and got[3] == ref[3]
        assert np.array_equal(got[2], ref[2])
    assert _run(device, preset, 2)[0] == ref[0]  # the default
    assert _run(oracle, preset, 2)[0] == ref[0]


def test_mill_blocks_bounds(device):
    s = Simulation(device, device.preset(device.params_default(), "realtime"))
    with pytest.raises(MillError):
        s.set_options(mill_blocks=17)
    s.set_options(mill_blocks=16)
    s.close()
