"""The C-ABI library without a GPU: it loads, exports every entry point include/millgpu.h
declares, its struct layouts match the bindings, and its host-only Params logic (params.rs,
presets.ts) agrees with the oracle field for field. No compute call is made here."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Backend, MillError

from helpers import params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "millgpu.h")).read()
    return sorted(set(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(device_lib):
    syms = header_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(device_lib.dll, s)]
    assert not missing, missing


def test_struct_layouts_match_bindings(device_lib, oracle_lib):
    assert device_lib.sizeof_params() == C.sizeof(capi.Params) == oracle_lib.sizeof_params()
    assert device_lib.sizeof_fluid_stats() == C.sizeof(capi.FluidStepStats)
    assert device_lib.sizeof_dem_stats() == C.sizeof(capi.DemStepStats)


def test_params_logic_matches_oracle(device, oracle):
    cases = [{}, {"mill.diameter_m": 0.6}, {"mill.speed_mode": capi.SPEED_PERCENT_CRITICAL, "mill.speed_value": 70.0},
             {"mill.diameter_m": 1.0, "media.ball_diameter_m": 0.010, "simulation.coarse_graining_mode": capi.CG_AUTO},
             {"media.ball_diameter_m": 0.3, "media.fill_fraction": 0.3, "simulation.coarse_graining_mode": capi.CG_MANUAL,
              "simulation.coarse_graining_k": 2.0}, {"media.fill_fraction": 0.4}, {"mill.direction": capi.DIR_CW}]
    for preset in (None, "realtime", "balanced", "accuracy", "impact_stats"):
        for kw in cases:
            pd, po = params(device, preset, **kw), params(oracle, preset, **kw)
            assert bytes(pd) == bytes(po)
            assert device.derived(pd).to_dict() == oracle.derived(po).to_dict()


def test_validation_messages_match_oracle(device, oracle):
    for field, value in [("mill.diameter_m", 0.0), ("media.fill_fraction", 1.5), ("slurry.wettability", 2.0),
                         ("simulation.resolution", 2), ("media.friction_ball_wall_static", 0.0)]:
        with pytest.raises(MillError) as ed:
            device.validate(params(device, **{field: value}))
        with pytest.raises(MillError) as eo:
            oracle.validate(params(oracle, **{field: value}))
        assert str(ed.value) == str(eo.value)


def test_no_device_fails_loudly_without_gpu(device):
    """On a machine without a CUDA device the library refuses to run (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(MillError) as e:
        from milldynamics3_b200.sim import Simulation
        Simulation(device, device.params_default())
    assert e.value.code == capi.MG_ERR_NO_DEVICE
    with pytest.raises(MillError) as e:
        from milldynamics3_b200.batch import Batch
        Batch(device, [device.params_default()] * 2)
    assert e.value.code == capi.MG_ERR_NO_DEVICE
    with pytest.raises(MillError) as e:
        from milldynamics3_b200.server import Server
        Server(device)
    assert e.value.code == capi.MG_ERR_NO_DEVICE
