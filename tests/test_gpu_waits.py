"""The device's bounded waits run out and come back as errors, with nothing hung.

The sub-step kernel has two kinds of waits: a single mill's block waits for its helper blocks at
the end of each shared per-ball phase, and in the drag and buoyancy sweeps a ball waits for the
earlier balls that share one of its fluid particles. Each wait has a bound; when it runs out the
kernel sets an error bit, stops the mill at its next check and releases the helper blocks, and
the host returns an error. Here the test options shorten the bounds to milliseconds and make a
wait that can never be satisfied: the mill's block waits for one more helper block than was
launched, or ball 0 of the drag sweep is never flagged done. Both are made on purpose and
bounded; the GPU context stays usable, and a fresh handle on default options then steps the
realtime mill bit for bit like the oracle.
"""
from __future__ import annotations

import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import MillError, Simulation

pytestmark = pytest.mark.gpu


def _realtime(b):
    return Simulation(b, b.preset(b.params_default(), "realtime"))


def _fresh_step_matches_oracle(device, oracle):
    sd, so = _realtime(device), _realtime(oracle)
    for _ in range(3):
        sd.step_fixed()
        so.step_fixed()
    assert sd.state_hash(True) == so.state_hash(True)
    sd.close()


def test_missing_helper_block_times_out_and_reports(device, oracle):
    s = _realtime(device)
    s.set_options(mill_blocks=4, test_wait_limit_us=2000, test_faults=1)
    with pytest.raises(MillError) as e:
        s.step_fixed()
    assert e.value.code == capi.MG_ERR_CUDA
    assert "stopped waiting for one another" in str(e.value)
    # the same handle steps again once the fault is gone
    s.set_options(mill_blocks=4)
    s.step_fixed()
    s.close()
    _fresh_step_matches_oracle(device, oracle)


def test_ball_never_flagged_done_times_out_and_reports(device, oracle):
    s = _realtime(device)
    s.set_options(test_wait_limit_us=500, test_faults=2)
    with pytest.raises(MillError) as e:
        s.step_fixed()
    assert e.value.code == capi.MG_ERR_STATE
    assert "bounded device wait ran out" in str(e.value)
    s.close()
    _fresh_step_matches_oracle(device, oracle)


def test_test_options_are_checked(device):
    s = _realtime(device)
    with pytest.raises(MillError):
        s.set_options(test_faults=4)
    with pytest.raises(MillError):
        s.set_options(test_wait_limit_us=20_000_000)
    s.close()
