"""The reference unit tests of tests/test_oracle_reference.py run through the CUDA library: the
same setups and assertions on the device, and, where the oracle finishes in seconds, the
returned quantities (impulses, velocities, energies, residuals, state hashes) equal to the
oracle's bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import scenarios_ref as R
from milldynamics3_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _canon(r):
    """Returned values in comparable form: a Simulation becomes its extended state hash."""
    if isinstance(r, Simulation):
        return ("hash", r.state_hash(True))
    if isinstance(r, (tuple, list)):
        return tuple(_canon(x) for x in r)
    if isinstance(r, dict):
        return tuple((k, _canon(v)) for k, v in sorted(r.items()))
    if isinstance(r, np.ndarray):
        return ("arr", r.dtype.str, r.shape, r.tobytes())
    if hasattr(r, "_fields_"):
        return ("struct", bytes(r))
    if isinstance(r, (float, np.floating)):
        return ("f", np.float64(r).tobytes())
    return r


@pytest.mark.parametrize("name", [
    "drag_matches_stokes_scaling",                       # pbf.rs:2677
    "drag_gains_form_drag",                              # pbf.rs:2743
    "drag_never_overshoots",                             # pbf.rs:2785
    "buoyancy_vertical_at_rest_inward_when_co_rotating",  # pbf.rs:2819
    "buoyancy_ignores_drum_rotation_for_a_still_pool",   # pbf.rs:2886
    "wall_drag_work",                                    # pbf.rs:2938
    "coupling_finds_neighbours_beyond_two_radii",        # pbf.rs:2985
    "hydrostatic_column",                                # pbf.rs:3032
    "viscosity_noop_at_zero",                            # pbf.rs:3133
    "viscosity_matters_between_100_and_200",             # pbf.rs:3149
    "viscosity_converges_at_high_viscosity_and_rotation",  # pbf.rs:3175
    "higher_viscosity_damps_more",                       # pbf.rs:3269
    "cohesion_two_particles",                            # pbf.rs:3463
    "adhesion_only_when_wettable",                       # coupling.rs:347
    "adhesion_range_is_capped",                          # coupling.rs:436
    "rolling_without_slip",                              # dem.rs:1334
    "lifter_wall_work",                                  # dem.rs:1382
    "energy_never_increases_in_still_drum",              # dem.rs:1784
    "dissipation_never_negative",                        # dem.rs:2130
    "steady_cascading_energy",                           # lib.rs:761
    "energy_budget_torque_readings",                     # lib.rs:1205
    "mixing_index_increases",                            # metrics.rs:888
    "mixing_index_weights_by_count",                     # metrics.rs:921
])
def test_reference_assertions_hold_on_the_device_and_match_the_oracle(device, oracle, name):
    rd = getattr(R, name)(device)
    ro = getattr(R, name)(oracle)
    assert _canon(rd) == _canon(ro), name


@pytest.mark.parametrize("viscosity", [50.0, 200.0])
def test_cascading_charge_clamp_rate(device, oracle, viscosity):
    # coupling.rs:788 and :806
    sd, rd = R.cascading_clamp_rate(device, viscosity)
    so, ro = R.cascading_clamp_rate(oracle, viscosity)
    assert rd == ro and sd.state_hash(True) == so.state_hash(True)


def test_low_fill_cataracting_charge_gains_no_energy(device):
    # coupling.rs:930
    R.low_fill_cataracting_energy(device)


def test_coupled_charge_gains_no_more_energy_than_the_wall_supplies(device):
    # coupling.rs:1149
    R.coupled_charge_energy(device)


def test_lifters_never_tunnel(device, oracle_lib):
    # dem.rs:2060 (the oracle measures the lifter SDF of the device's ball positions)
    R.lifters_never_tunnel(device, oracle_lib)


def test_cascading_charge_density_samples_match_the_oracle(device, oracle):
    # dem.rs:1968's run; its bounds are checked in the median (see the oracle test) and the
    # samples equal the oracle's
    over, mind = R.cascading_density_samples(device)
    assert (over, mind) == R.cascading_density_samples(oracle)
    assert sorted(over)[len(over) // 2] < 0.7 and min(mind) > 0.05 * 0.5


@pytest.mark.parametrize("name", ["wall_ccd_clamps_a_fast_ball",        # dem.rs:674-706
                                  "bingham_damps_more_than_newtonian",  # pbf.rs:2146-2153, 800-868
                                  "bingham_realtime_mill"])
def test_untested_branches_run_on_the_device_and_match_the_oracle(device, oracle, name):
    rd = getattr(R, name)(device)
    ro = getattr(R, name)(oracle)
    assert _canon(rd) == _canon(ro), name
