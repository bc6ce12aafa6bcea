"""Request server (mg_server_*): jobs admitted while others run, under a memory budget, give
exactly the results of the same mills stepped alone (and of the oracle)."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.batch import mix_params
from milldynamics3_b200.server import Server
from milldynamics3_b200.sim import Simulation

pytestmark = pytest.mark.gpu
FRAME = 1.0 / 60.0


def _small_jobs(backend, n, seed):
    ps, _ = mix_params(backend, 4 * n, seed=seed)
    d = [backend.derived(p) for p in ps]
    order = sorted(range(len(ps)), key=lambda i: d[i].eff_ball_count * d[i].effective_fluid_resolution ** 2)
    return [ps[i] for i in order[:n]]


def _alone(backend, p, frames):
    s = Simulation(backend, p)
    for _ in range(frames):
        s.step(FRAME)
    out = (s.state_hash(True), s.scalars().to_dict(), np.array(s.stress_histogram_rate()))
    s.close()
    return out


def _run_until_done(server, max_steps=200):
    ups = []
    for _ in range(max_steps):
        server.step()
        ups += server.poll()
        st = server.stats()
        if st.queued == 0 and st.active == 0:
            return ups
    raise AssertionError("server did not drain")


def test_jobs_in_the_mix_match_jobs_alone(device):
    ps = _small_jobs(device, 5, seed=11)
    frames = [3, 1, 4, 2, 3]
    server = Server(device)
    ids = {}
    for k in range(3):
        ids[server.submit(ps[k], frames[k] * FRAME)] = k
    server.step()
    ups = server.poll()
    for k in (3, 4):  # arrive while the first three are running
        ids[server.submit(ps[k], frames[k] * FRAME)] = k
    ups += _run_until_done(server)
    final = {u.job_id: u for u in ups if u.state != capi.JOB_RUNNING}
    assert set(final) == set(ids)
    for jid, k in ids.items():
        u = final[jid]
        assert u.state == capi.JOB_FINISHED and u.frames_done == frames[k]
        h, sc, hist = _alone(device, ps[k], frames[k])
        assert u.state_hash == h, f"job {k}"
        assert u.scalars.to_dict() == sc, f"job {k} scalars"
        assert np.array_equal(np.array(u.stress_histogram_rate), hist), f"job {k} histogram"
    # streamed progress: one RUNNING update per job and frame before the last
    for jid, k in ids.items():
        running = [u.frames_done for u in ups if u.job_id == jid and u.state == capi.JOB_RUNNING]
        assert running == list(range(1, frames[k]))
    server.close()


def test_job_matches_oracle(device, oracle):
    p = _small_jobs(device, 1, seed=13)[0]
    server = Server(device)
    jid = server.submit(p, 2 * FRAME)
    ups = _run_until_done(server)
    u = [x for x in ups if x.job_id == jid and x.state == capi.JOB_FINISHED][0]
    so = Simulation(oracle, p)
    so.step(FRAME)
    so.step(FRAME)
    assert u.state_hash == so.state_hash(True)
    server.close()


def test_admission_waits_for_memory_and_cancel(device):
    import ctypes as C
    ps = _small_jobs(device, 4, seed=17)[::-1]  # the two largest first, so the others fit after them
    fps = []
    for p in ps[:2]:
        probe = Simulation(device, p)
        fp = C.c_uint64()
        device.lib.sim_footprint(probe.h, C.byref(fp))
        fps.append(fp.value)
        probe.close()
    # room for the two oldest jobs only: the third waits until one of them retires
    budget = fps[0] + fps[1]
    server = Server(device, memory_budget_bytes=budget)
    ids = [server.submit(p, 2 * FRAME) for p in ps]
    server.step()
    st = server.stats()
    assert st.active == 2 and st.queued == 2 and st.device_bytes_in_use <= budget
    server.cancel(ids[-1])  # still queued: leaves at once
    ups = server.poll() + _run_until_done(server)
    final = {u.job_id: u for u in ups if u.state != capi.JOB_RUNNING}
    assert final[ids[-1]].state == capi.JOB_CANCELLED
    for k, jid in enumerate(ids[:-1]):
        assert final[jid].state == capi.JOB_FINISHED
        assert final[jid].state_hash == _alone(device, ps[k], 2)[0], f"job {k}"
    assert server.stats().device_bytes_in_use == 0
    server.close()


def _run_until_sweep_done(srv, sid, n, max_steps=5000):
    for _ in range(max_steps):
        st, done, res, mean, se = srv.sweep_result(sid, n)
        if st not in (capi.JOB_QUEUED, capi.JOB_RUNNING):
            return st, done, res, mean, se
        srv.step()
        srv.poll()
    raise AssertionError("sweep did not finish")


def test_sweep_job_matches_seed_sweep_and_oracle(device, oracle):
    from milldynamics3_b200 import seeds
    p = device.preset(device.params_default(), "realtime")
    srv = Server(device)
    other = srv.submit(mix_params(device, 1, seed=9)[0][0], 0.5)   # an ordinary job in the same launches
    sid = srv.submit_sweep(p, 3, 0.25, 1.0)
    st, done, res, mean, se = _run_until_sweep_done(srv, sid, 3)
    assert st == capi.JOB_FINISHED and done == 3 and other > 0
    ref = seeds.run_seeds(device, p, [1, 2, 3], 0.25, 1.0)
    for r, d in zip(res, ref):
        assert r.seed == d.seed and r.window_s == d.window_s
        assert list(r.values) == d.values and r.power_drift_rel_per_rev == d.power_drift_rel_per_rev
    po = oracle.preset(oracle.params_default(), "realtime")
    assert list(res[0].values) == seeds.run_seed(oracle, po, 1, 0.25, 1.0).values
    c = seeds.combine(device, ref)
    assert mean == c.mean and se == c.std_err


def test_sweep_job_rules_and_cancel(device):
    from milldynamics3_b200.sim import MillError
    srv = Server(device)
    p = device.preset(device.params_default(), "realtime")
    for bad in [(0, 0.0, 1.0), (capi.SWEEP_MAX_SEEDS + 1, 0.0, 1.0), (2, -1.0, 1.0), (2, 0.0, 1.5), (2, 0.0, 0.0)]:
        with pytest.raises(MillError):
            srv.submit_sweep(p, *bad)
    q = device.params_default()
    q.mill.speed_value = 0.0
    with pytest.raises(MillError):
        srv.submit_sweep(q, 2, 0.0, 1.0)
    cg = device.params_default()
    cg.mill.diameter_m = 1.0
    cg.media.ball_diameter_m = 0.02
    cg.simulation.max_balls = 300
    cg.simulation.coarse_graining_mode = capi.CG_AUTO
    device.validate(cg)
    if device.derived(cg).eff_scale_factor > 1.0:
        with pytest.raises(MillError):
            srv.submit_sweep(cg, 2, 0.0, 1.0)
    sid = srv.submit_sweep(p, 2, 0.0, 1.0)
    srv.step()
    srv.cancel(sid)
    for _ in range(3):
        srv.step()
    st, done, res, _, _ = srv.sweep_result(sid, 2)
    assert st == capi.JOB_CANCELLED and res is None
    assert srv.stats().active == 0


def test_sweep_that_fails_cancels_its_other_seeds_and_release_forgets_it(device):
    from milldynamics3_b200.sim import MillError
    p = device.preset(device.params_default(), "realtime")
    # a budget no mill fits: the first seed fails at admission (nothing running could free memory),
    # and its two siblings leave as cancelled instead of waiting in the queue
    srv = Server(device, memory_budget_bytes=1 << 20)
    sid = srv.submit_sweep(p, 3, 0.0, 1.0)
    srv.step()
    ups = srv.poll()
    states = sorted(u.state for u in ups)
    assert states == sorted([capi.JOB_FAILED, capi.JOB_CANCELLED, capi.JOB_CANCELLED])
    st, done, res, _, _ = srv.sweep_result(sid, 3)
    assert st == capi.JOB_FAILED and done == 0 and res is None
    s = srv.stats()
    assert s.active == 0 and s.queued == 0
    srv.release_sweep(sid)
    with pytest.raises(MillError):
        srv.sweep_result(sid, 3)
    srv.close()
    # releasing a running sweep cancels its seeds before the next frame
    srv = Server(device)
    sid = srv.submit_sweep(p, 2, 0.0, 1.0)
    srv.step()
    assert srv.stats().active == 2
    srv.release_sweep(sid)
    srv.step()
    assert srv.stats().active == 0
    with pytest.raises(MillError):
        srv.release_sweep(sid)
    srv.close()
