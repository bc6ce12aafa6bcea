"""The tolerance probe on the device library (every run of a frame window a mill of one batch)
gives the oracle's per-config means and standard errors, run by run."""
from __future__ import annotations

import math

import pytest

from milldynamics3_b200 import tolerance as tp

pytestmark = pytest.mark.gpu


def _same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


def test_device_probe_equals_oracle(device, oracle):
    only = ["ship_fast", "ship_acc", "ship_v50"]
    kw = dict(seeds=2, settle_revs=0.02, measure_revs=0.06, only=only)
    dev = tp.run_all(device, batched=True, **kw)
    orc = tp.run_all(oracle, batched=False, **kw)
    assert dev.keys() == orc.keys()
    for key in dev:
        if key[1] == "ms_per_frame":
            continue
        assert _same(dev[key][0], orc[key][0]) and _same(dev[key][1], orc[key][1]), (key, dev[key], orc[key])
    assert tp.compare(orc, dev, lambda _: None) == 0
