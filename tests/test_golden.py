"""The committed fixtures (tests/golden/oracle_states.json, written by tests/golden/make_golden.py
from the oracle) for the realtime mill, its 300-disc variant, a balls-only 500-disc mill and a
large 5,000-disc / 12.7k-fluid mill at two viscosities: the oracle must still reproduce them (CPU)
and the device must reproduce them bit for bit (GPU). Integer and bit-pattern results, so the
tolerance is exact equality (the state hash covers every position, velocity, angle and spin)."""
from __future__ import annotations

import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import cases  # noqa: E402

FIXTURES = json.load(open(os.path.join(HERE, "golden", "oracle_states.json")))


@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_oracle_reproduces_fixture(oracle, name):
    assert cases.run_case(oracle, name) == FIXTURES[name]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIXTURES))
def test_device_reproduces_fixture(device, name):
    assert cases.run_case(device, name) == FIXTURES[name]
