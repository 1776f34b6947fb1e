"""Serving loop (rf_server_*): continuous batching of independent suspensions.

Each request's result must be the same alone and in the mix: bit-identical
fiber state and velocities when the same server configuration runs it alone
and beside other requests (all reductions have a fixed order, no atomics),
and within 1e-5 relative of a stand-alone Simulation (whose cooperative
Krylov grids may be wider, which changes the order of the FP64 dot-product
partials only).
"""
import numpy as np
import pytest

from rigidfibers_b200.generate import request_layout, serving_requests

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _cfg(req, **kw):
    from rigidfibers_b200 import Config
    base = dict(slenderness=req["slenderness"], precision="mixed_bf16", refinement_tolerance=1e-6)
    base.update(kw)
    return Config(**base)


MIX = [dict(precision="mixed_bf16"), dict(precision="mixed_fp16"), dict(precision="fp32"),
       dict(precision="fp32", solver="bicgstab"), dict(precision="fp32", solver="direct"),
       dict(precision="fp32", integration="analytical")]


def _requests():
    reqs = serving_requests(count=12, seed=7, n_min=16, n_max=300, steps_min=2, steps_max=5)
    return [(r, MIX[i % len(MIX)]) for i, r in enumerate(reqs)]


def test_result_alone_equals_result_in_the_mix():
    from rigidfibers_b200 import Simulation
    from rigidfibers_b200.server import Server
    reqs = _requests()
    layouts = [request_layout(r) for r, _ in reqs]
    alone = []
    with Server(max_active=4) as srv:
        for (r, kw), (p, o) in zip(reqs, layouts):
            rid = srv.submit(_cfg(r, **kw), p, o, r["nsteps"])
            assert srv.wait(rid) == "done"
            alone.append(srv.result(rid))
    with Server(max_active=4) as srv:
        ids = [srv.submit(_cfg(r, **kw), p, o, r["nsteps"]) for (r, kw), (p, o) in zip(reqs, layouts)]
        srv.drain()
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["peak_active"] > 1           # the requests did overlap
        assert st["p99_step_ms"] >= st["p50_step_ms"] > 0
        for rid, a in zip(ids, alone):
            got = srv.result(rid)
            for k in range(4):
                assert np.array_equal(got[k], a[k]), (rid, k)
            assert got[4]["steps_done"] == a[4]["steps_done"]
    # and against a lone Simulation of the same request
    for (r, kw), (p, o), a in list(zip(reqs, layouts, alone))[:4]:
        sim = Simulation(_cfg(r, **kw), p, o)
        sim.run(r["nsteps"])
        pos, ori = sim.state()
        tv, rv = sim.velocities()
        sim.close()
        assert _rel(a[0], pos) <= 1e-5 and _rel(a[1], ori) <= 1e-5
        assert _rel(a[2], tv) <= 1e-5 and _rel(a[3], rv) <= 1e-5


def test_admission_respects_the_memory_budget():
    from rigidfibers_b200.server import Server, device_bytes
    reqs = serving_requests(count=10, seed=3, n_min=100, n_max=400, steps_min=1, steps_max=2)
    need = [device_bytes(_cfg(r), r["n"]) for r in reqs]
    budget = int(max(need) * 1.5)
    with Server(max_active=8, hbm_budget_bytes=budget) as srv:
        for r in reqs:
            p, o = request_layout(r)
            srv.submit(_cfg(r), p, o, r["nsteps"])
        srv.drain()
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["peak_bytes"] <= budget
    assert st["peak_active"] < 8


def test_request_larger_than_budget_is_refused():
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.server import Server, device_bytes
    r = serving_requests(count=1, seed=1, n_min=200, n_max=200)[0]
    p, o = request_layout(r)
    with Server(max_active=2, hbm_budget_bytes=device_bytes(_cfg(r), r["n"]) - 1) as srv:
        with pytest.raises(C.RigidFibersError) as e:
            srv.submit(_cfg(r), p, o, 3)
        assert e.value.status == C.RF_E_OOM


def test_cancel_stops_a_running_request():
    from rigidfibers_b200.server import Server
    r = serving_requests(count=1, seed=2, n_min=400, n_max=400)[0]
    p, o = request_layout(r)
    with Server(max_active=1) as srv:
        long_id = srv.submit(_cfg(r), p, o, 100000)
        queued_id = srv.submit(_cfg(r), p, o, 5)
        srv.cancel(queued_id)
        import time
        t0 = time.time()
        while srv.poll(long_id)[1] < 2 and time.time() - t0 < 60:
            time.sleep(0.01)
        srv.cancel(long_id)
        assert srv.wait(long_id) == "cancelled"
        assert srv.wait(queued_id) == "cancelled"
        done = srv.poll(long_id)[1]
        assert 2 <= done < 100000
        pos, ori, tv, rv, st = srv.result(long_id)
        assert st["steps_done"] == done and np.isfinite(pos).all()


def test_invalid_request_is_refused_at_submit():
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.server import Server
    r = serving_requests(count=1, seed=4, n_min=30, n_max=30)[0]
    p, o = request_layout(r)
    bad = _cfg(r, precision="mixed_bf16", integration="analytical")   # mixed needs numerical integration
    with Server(max_active=2) as srv:
        with pytest.raises(C.RigidFibersError) as e:
            srv.submit(bad, p, o, 2)
        assert e.value.status == C.RF_E_INPUT


def test_failed_request_reports_its_status():
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.server import Server
    r = serving_requests(count=1, seed=4, n_min=30, n_max=30)[0]
    p, o = request_layout(r)
    pnan = p.copy()
    pnan[3, 1] = np.nan
    with Server(max_active=2) as srv:
        rid = srv.submit(_cfg(r), pnan, o, 2)
        ok = srv.submit(_cfg(r), p, o, 2)
        assert srv.wait(rid) == "failed"
        assert srv.wait(ok) == "done"
        with pytest.raises(C.RigidFibersError) as e:
            srv.result(rid)
        assert e.value.status == C.RF_E_NAN


def _serve_with_graph_mode(graphs):
    from rigidfibers_b200 import Config
    from rigidfibers_b200.server import Server
    reqs = serving_requests(count=4, seed=19, n_min=16, n_max=200, steps_min=3, steps_max=6)
    out = []
    with Server(max_active=2, use_cuda_graphs=graphs, reserve_bytes=1 << 28) as srv:
        ids = [srv.submit(Config(precision="mixed_bf16"), *request_layout(r), r["nsteps"]) for r in reqs]
        srv.drain(timeout=300)
        for r, rid in zip(reqs, ids):
            t = srv.step_times(rid)
            assert len(t) == r["nsteps"] and (t > 0).all()
            out.append(srv.result(rid)[:2])
        st = srv.stats()
        assert st["p50_setup_ms"] > 0 and st["p99_setup_ms"] >= st["p50_setup_ms"]
        assert st["completed"] == len(reqs)
    return out


def test_step_times_setup_and_graph_modes():
    """rf_server_step_times returns one wall time per step of a finished
    request; the server's set-up percentiles cover handle creation and, with
    whole-step graphs (mode 1), building them before the first step; the
    results of mode 1 and mode 2 (restart cycles) are the same bit for bit."""
    a = _serve_with_graph_mode(1)
    b = _serve_with_graph_mode(2)
    for (pa, oa), (pb, ob) in zip(a, b):
        assert np.array_equal(pa, pb) and np.array_equal(oa, ob)
