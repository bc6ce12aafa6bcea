"""The f64 mode of the viscosity solve (MgOptions.cg_fp64 = 1: inner products and residual norms
in f64) against the oracle in its f64 mode. The device forms those f64 sums as block trees, the
oracle left to right, so the two agree to rounding in the solve, not bit for bit: one sub-step is
checked against the specification's single-step tolerance, 1e-5 relative to each array's largest
magnitude, at water viscosity and at 0.1 Pa s (several CG iterations)."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200.sim import Simulation

from helpers import params

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max() if b.size else 0.0, 1e-30)
    return np.abs(a - b).max() / scale if a.size else 0.0


@pytest.mark.parametrize("viscosity", [1e-3, 1e-1])
def test_fp64_solve_matches_oracle_fp64(device, oracle, viscosity):
    sims = []
    for b in (device, oracle):
        s = Simulation(b, params(b, "realtime", **{"slurry.viscosity_pa_s": viscosity}))
        s.set_options(cg_fp64=1)
        s.step_fixed()
        sims.append(s)
    sd, so = sims
    bd, bo = sd.balls(), so.balls()
    fd, fo = sd.fluid(), so.fluid()
    for k in ("x", "v"):
        assert _rel(fd[k], fo[k]) <= REL_TOL, f"fluid.{k}"
        assert _rel(bd[k], bo[k]) <= REL_TOL, f"balls.{k}"
    assert _rel(bd["omega"], bo["omega"]) <= REL_TOL
    # the solve's iteration count is an integer outcome of the same tolerance test
    assert sd.last_step_stats()[0].viscosity_iterations == so.last_step_stats()[0].viscosity_iterations


def test_fp64_and_f32_modes_are_close(device):
    """Switching the solve's reductions to f64 moves one sub-step by rounding only."""
    out = []
    for mode in (0, 1):
        s = Simulation(device, params(device, "realtime", **{"slurry.viscosity_pa_s": 1e-1}))
        s.set_options(cg_fp64=mode)
        s.step_fixed()
        out.append(s.fluid()["v"])
    assert _rel(out[1], out[0]) <= 1e-4
