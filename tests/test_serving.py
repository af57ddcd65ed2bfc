"""The serving loop: simulations of two model structures submitted at
different times, admitted by a device-memory budget, packed and stepped
together, leaving when done.  Every result must be bit-identical to the same
simulation run alone in a Session of the same precision.
"""
import numpy as np
import pytest

import grasph_b200 as G
from grasph_b200 import scenarios
from gc_helpers import make_backend

pytestmark = pytest.mark.gpu


def _requests():
    cols = scenarios.batched_columns(count=4, seed=3, nmin=300, nmax=2000, dx=0.002)
    out = [(lf, m, 37 + 11 * k) for k, (lf, m) in enumerate(cols)]
    for k, (nx, ny, nz) in enumerate([(6, 4, 8), (8, 5, 10)]):
        lf, m = scenarios.dambreak_3d(nx=nx, ny=ny, nz=nz, dx=0.05, tank=(1.0, 0.5, 1.0))
        out.append((lf, m, 45 + 7 * k))
    return out


def _alone(k, prec):
    lf, meta, nsteps = _requests()[k]
    s = G.Session([lf], backend=make_backend("cuda"), precision=prec)
    s.push()
    s.step(nsteps, meta["cfl"])
    s.pull(with_ghosts=False)
    return lf


@pytest.mark.parametrize("prec", [G.PRECISION_FP64, G.PRECISION_FP32_COMPENSATED])
def test_served_results_equal_alone(prec):
    reqs = _requests()
    srv = G.Server(round_steps=16, precision=prec, hbm_budget=2 * 10**9)
    ids = {}
    # staggered arrivals: two requests, a round, the rest one per round
    order = [0, 4, 1, 2, 5, 3]
    for k in order[:2]:
        lf, meta, n = reqs[k]
        ids[k] = srv.submit(lf, n, meta["cfl"])
    pending = order[2:]
    rounds = 0
    while True:
        srv.pump()
        rounds += 1
        if pending:
            k = pending.pop(0)
            lf, meta, n = reqs[k]
            ids[k] = srv.submit(lf, n, meta["cfl"])
        st = [srv.poll(r)["state"] for r in ids.values()]
        assert G.Server.FAILED not in st
        if not pending and all(x == G.Server.DONE for x in st):
            break
        assert rounds < 200
    stats = srv.stats()
    assert stats["repacks"] >= 3 and stats["running"] == 0 and stats["queued"] == 0
    for k, req in ids.items():
        info = srv.poll(req)
        assert info["steps_done"] == reqs[k][2]
        assert info["t_submit"] <= info["t_admit"] <= info["t_done"]
        got = srv.fetch(req)
        ref = _alone(k, prec)
        for sg, sr in zip(got.systems, ref.systems):
            for name, _ in sg.particle_fields():
                assert np.array_equal(getattr(sg, name), getattr(sr, name), equal_nan=True), \
                    f"request {k}: {sg.name}.{name} differs from the run alone"
        srv.release(req)


def test_budget_holds_requests_back():
    reqs = _requests()
    lf0, meta0, n0 = reqs[0]
    srv = G.Server(round_steps=8, hbm_budget=1)  # nothing fits: every request fails
    r = srv.submit(lf0, n0, meta0["cfl"])
    srv.pump()
    assert srv.poll(r)["state"] == G.Server.FAILED


def _estimate(lf, meta, n):
    """A request's device-memory estimate, as the server reserves it."""
    srv = G.Server(round_steps=1, hbm_budget=10**12)
    r = srv.submit(lf, n, meta["cfl"])
    srv.pump()
    est = srv.stats()["device_bytes_reserved"]
    srv.close()
    return est


def test_request_waits_for_budget_then_runs():
    """Two requests that fit the budget one at a time but not together: the
    second stays queued while the first runs, is admitted after the first
    finishes, and its result still equals the run alone."""
    reqs = _requests()
    (la, ma, na), (lb, mb, nb) = reqs[4], reqs[5]
    ea, eb = _estimate(*_requests()[4]), _estimate(*_requests()[5])
    assert ea > 0 and eb > 0
    srv = G.Server(round_steps=8, hbm_budget=max(ea, eb) + min(ea, eb) // 2)
    ra = srv.submit(la, na, ma["cfl"])
    rb = srv.submit(lb, nb, mb["cfl"])
    srv.pump()
    assert srv.poll(ra)["state"] in (G.Server.RUNNING, G.Server.DONE)
    assert srv.poll(rb)["state"] == G.Server.QUEUED
    waited = 0
    while srv.poll(ra)["state"] != G.Server.DONE:
        assert srv.poll(rb)["state"] == G.Server.QUEUED
        srv.pump()
        waited += 1
        assert waited < 100
    rounds = 0
    while srv.poll(rb)["state"] != G.Server.DONE:
        srv.pump()
        rounds += 1
        assert rounds < 100
    a, b = srv.poll(ra), srv.poll(rb)
    assert b["t_admit"] >= a["t_done"] and waited >= 1
    got = srv.fetch(rb)
    ref = _alone(5, G.PRECISION_FP32_COMPENSATED)
    for sg, sr in zip(got.systems, ref.systems):
        for name, _ in sg.particle_fields():
            assert np.array_equal(getattr(sg, name), getattr(sr, name), equal_nan=True), f"{sg.name}.{name}"
    st = srv.stats()
    assert st["repacks"] >= 2 and st["repack_seconds"] > 0.0 and st["repack_instances"] >= 2


def test_failing_request_is_retried_alone_and_isolated():
    """A request with a non-finite position makes its batch's step fail,
    whichever of the batch's requests caused it.  The server then runs the
    batch's requests again from their submitted state, each in a batch of
    its own: only the bad request fails, and the others finish with the
    results of the same simulation run alone."""
    reqs = _requests()[:3]  # three columns: one structure, one batch
    bad_lf, _, _ = _requests()[1]
    bad_lf.systems[0].x[0, 0] = np.nan
    srv = G.Server(round_steps=8, precision=G.PRECISION_FP64, hbm_budget=2 * 10**9)
    ids = []
    for k, (lf, meta, n) in enumerate(reqs):
        ids.append(srv.submit(bad_lf if k == 1 else lf, n, meta["cfl"]))
    rounds = 0
    while any(srv.poll(r)["state"] in (G.Server.QUEUED, G.Server.RUNNING) for r in ids):
        srv.pump()
        rounds += 1
        assert rounds < 400
    assert [srv.poll(r)["state"] for r in ids] == [G.Server.DONE, G.Server.FAILED, G.Server.DONE]
    assert srv.stats()["retries"] >= 3
    for k in (0, 2):
        got = srv.fetch(ids[k])
        ref = _alone(k, G.PRECISION_FP64)
        for sg, sr in zip(got.systems, ref.systems):
            for name, _ in sg.particle_fields():
                assert np.array_equal(getattr(sg, name), getattr(sr, name), equal_nan=True), \
                    f"request {k}: {sg.name}.{name}"
