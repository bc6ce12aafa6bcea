"""The launch-shape autotuner on the device: it times the candidates, checks that they all leave
the same state bits, records the fastest per size bucket, and its table round-trips."""
from __future__ import annotations

import json

import pytest

from milldynamics3_b200 import autotune, workloads
from milldynamics3_b200.batch import mix_params

pytestmark = pytest.mark.gpu


def test_mill_tuning_picks_a_candidate_and_keeps_results(device, tmp_path):
    at = autotune.Autotuner(device, frames=2)
    p, balls = workloads.realtime(device)
    cands = autotune.MILL_CANDIDATES[:3]
    t = at.tune_mill(p, balls, candidates=cands)
    assert t.options in cands and t.ms > 0 and len(t.timings) == 3
    key = autotune.bucket(794, 407)
    assert at.table[key]["options"] == t.options
    path = tmp_path / "tuned.json"
    at.save(str(path))
    other = autotune.Autotuner(device)
    other.load(str(path))
    assert other.mill_options(p, balls) == t.options
    assert json.loads(path.read_text())[key]["ms"] == t.ms


def test_batch_tuning_compares_every_mill(device):
    ps, _ = mix_params(device, 12, seed=4)
    at = autotune.Autotuner(device, frames=1)
    t = at.tune_batch(ps)
    assert t.options in autotune.BATCH_CANDIDATES and set(t.timings) == {
        json.dumps(c, sort_keys=True) for c in autotune.BATCH_CANDIDATES}
