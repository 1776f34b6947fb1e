"""Packed solves of many small suspensions: rf_solve_packed / rf_step_packed
(one thread-block cluster per suspension) and the server's pack.

Bounds (written here): the packed solution within 1e-5 relative of rf_solve's
(both run GMRES-IR to a relative residual of 1e-6; only the summation order
differs) and within 1e-4 of the FP64 oracle's direct solve; a suspension's
result bit for bit the same alone and in a pack.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rigidfibers_b200.generate import sphere_layout

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _layout(n, seed):
    # the serving workload's density: circumscribed-sphere volume fraction 1 %
    return sphere_layout(n, max(1.5, (100.0 * n) ** (1.0 / 3.0)), 0.2, seed=seed)


def _sim(pos, ori, **kw):
    from rigidfibers_b200 import Config, Simulation
    return Simulation(Config(**kw), pos, ori)


@pytest.mark.parametrize("prec", ["mixed_fp16", "mixed_bf16"])
@pytest.mark.parametrize("n", [1, 7, 16, 33, 100, 128, 200, 256])
def test_packed_solve_matches_rf_solve_and_fp64(prec, n):
    from rigidfibers_b200.simulation import solve_packed
    pos, ori = _layout(n, 100 + n)
    a = _sim(pos, ori, precision=prec)
    a.assembleSystem()
    a.solveSystem()
    xa = a.solution()
    b = _sim(pos, ori, precision=prec)
    b.assembleSystem()
    solve_packed([b])
    xb = b.solution()
    st = b.stats()
    assert st["relative_residual"] <= 1e-6
    assert _rel(xb, xa) <= 1e-5
    A64, b64 = O.assemble(pos, ori, O.Params(), False, np.float64)
    x64 = np.linalg.solve(A64, b64) if n > 1 else np.zeros_like(b64)
    assert _rel(xb, x64) <= 1e-4
    if n > 1:
        assert st["iterations"] >= 1 and st["refinement_steps"] >= 1


def test_member_is_the_same_alone_and_in_a_pack():
    from rigidfibers_b200.simulation import solve_packed, step_packed
    lays = {"a": (_layout(40, 1), dict(precision="mixed_bf16")),
            "b": (_layout(100, 2), dict(precision="mixed_bf16", slenderness=0.005)),
            "c": (_layout(7, 3), dict(precision="mixed_bf16"))}
    alone = _sim(*lays["a"][0], **lays["a"][1])
    alone.assembleSystem()
    solve_packed([alone])
    x_alone = alone.solution()
    mix = {k: _sim(*v[0], **v[1]) for k, v in lays.items()}
    for s in mix.values():
        s.assembleSystem()
    solve_packed([mix["b"], mix["a"], mix["c"]])
    assert np.array_equal(mix["a"].solution(), x_alone)
    # whole steps: three of them, alone and beside two others
    one = _sim(*lays["a"][0], **lays["a"][1])
    many = [_sim(*lays[k][0], **lays[k][1]) for k in ("c", "a", "b")]
    for t in range(3):
        assert step_packed([one], [t]) == [0]
        assert step_packed(many, [t, t, t]) == [0, 0, 0]
    p1, o1 = one.state()
    p2, o2 = many[1].state()
    assert np.array_equal(p1, p2) and np.array_equal(o1, o2)


def test_member_is_the_same_for_every_cluster_size():
    """A member's packed solve is the same bits whatever cluster the pack's
    plan gives it: alone a 128-fiber suspension runs on 8 CTAs, a 64-fiber one
    on 4 and a 256-fiber one on 8; beside 148 other members (more members than
    multiprocessors) the first two run on one CTA and the third on two."""
    import ctypes
    import torch
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.simulation import solve_packed
    lib = C.load()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    fibers = [128, 64, 256] + [16] * max(148, sms - 2)

    def plan(fs):
        c = (ctypes.c_int * len(fs))()
        assert lib.rf_debug_pack_plan((ctypes.c_int * len(fs))(*fs), len(fs), sms, c) == C.RF_OK
        return list(c)

    assert plan([128]) == [8] and plan([64]) == [4] and plan([256]) == [8]
    assert plan(fibers)[:3] == [1, 1, 2]
    lays = [_layout(n, 300 + k) for k, n in enumerate(fibers)]
    alone = []
    for k in range(3):
        a = _sim(*lays[k], precision="mixed_fp16")
        a.assembleSystem()
        solve_packed([a])
        alone.append((a.solution(), a.stats()["iterations"]))
        a.close()
    sims = [_sim(*lay, precision="mixed_fp16") for lay in lays]
    for s in sims:
        s.assembleSystem()
    solve_packed(sims)
    for k in range(3):
        assert np.array_equal(sims[k].solution(), alone[k][0]), fibers[k]
        assert sims[k].stats()["iterations"] == alone[k][1]
    for s in sims:
        s.close()


def test_non_finite_member_of_a_clustered_pack_fails_alone():
    """A member whose positions hold a NaN (a 128-fiber suspension, on a
    cluster of CTAs) reports RF_E_NAN from rf_step_packed; the pack's other
    members step exactly as they do alone."""
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.simulation import step_packed
    pb, ob = _layout(128, 41)
    pb = pb.copy()
    pb[5, 0] = np.nan
    good = [_layout(64, 42), _layout(20, 43)]
    alone = []
    for lay in good:
        a = _sim(*lay, precision="mixed_bf16")
        assert step_packed([a], [0]) == [0]
        alone.append(a.state())
        a.close()
    sims = [_sim(pb, ob, precision="mixed_bf16")] + [_sim(*lay, precision="mixed_bf16") for lay in good]
    codes = step_packed(sims, [0, 0, 0])
    assert codes[0] == C.RF_E_NAN and codes[1:] == [0, 0]
    for sm, (pa, oa) in zip(sims[1:], alone):
        p, o = sm.state()
        assert np.array_equal(p, pa) and np.array_equal(o, oa)
    for sm in sims:
        sm.close()


def test_packed_steps_follow_rf_step():
    from rigidfibers_b200.simulation import step_packed
    pos, ori = _layout(60, 9)
    ref = _sim(pos, ori, precision="mixed_fp16")
    pk = _sim(pos, ori, precision="mixed_fp16")
    for t in range(2):
        ref.step(t)
        assert step_packed([pk], [t]) == [0]
    for a, b in zip(pk.state(), ref.state()):
        assert _rel(a, b) <= 1e-6
    for a, b in zip(pk.velocities(), ref.velocities()):
        assert _rel(a, b) <= 1e-5
    st = pk.stats()
    assert st["ms_solve_system"] > 0 and st["ms_assemble_system"] > 0


def test_packed_step_kernels_match_the_single_suspension_stages():
    """rf_step_packed's packed assembly, velocities and update (a few launches
    per pack) against the single-suspension stages around the same packed
    solve: rf_assemble, rf_solve_packed, rf_update_velocities and
    rf_update_fibers give the same state and velocities bit for bit.  The pack
    holds three groups (FP16 and BF16 storage, two slendernesses); its first
    member reports the pack's launches: the solve plus four per group."""
    from rigidfibers_b200.simulation import solve_packed, step_packed
    cfgs = [dict(precision="mixed_bf16"), dict(precision="mixed_fp16"),
            dict(precision="mixed_bf16", slenderness=0.005), dict(precision="mixed_fp16")]
    sizes = [1, 33, 128, 70]
    lays = [_layout(n, 40 + k) for k, n in enumerate(sizes)]
    staged = [_sim(*lay, **c) for lay, c in zip(lays, cfgs)]
    packed = [_sim(*lay, **c) for lay, c in zip(lays, cfgs)]
    for t in range(3):
        for s in staged:
            s.assembleSystem()
            solve_packed([s])
            s.updateVelocities()
            s.updateFibers(t == 0)
        assert step_packed(packed, [t] * len(packed)) == [0] * len(packed)
        for a, b in zip(staged, packed):
            for u, v in zip(a.state() + a.velocities(), b.state() + b.velocities()):
                assert np.array_equal(u, v)
    st = packed[0].stats()
    assert st["kernel_launches"] == 1 + 4 * 3
    assert packed[1].stats()["kernel_launches"] == 0
    assert st["ms_assemble_system"] > 0 and st["ms_solve_system"] > 0 and st["ms_update_velocities"] > 0


def test_packed_solve_refuses_what_it_does_not_take():
    from rigidfibers_b200 import _capi as C
    from rigidfibers_b200.simulation import solve_packed
    pos, ori = _layout(20, 5)
    fp32 = _sim(pos, ori)
    fp32.assembleSystem()
    with pytest.raises(C.RigidFibersError) as e:
        solve_packed([fp32])
    assert e.value.status == C.RF_E_UNSUPPORTED
    big = _sim(*_layout(257, 6), precision="mixed_bf16")
    big.assembleSystem()
    with pytest.raises(C.RigidFibersError) as e:
        solve_packed([big])
    assert e.value.status == C.RF_E_UNSUPPORTED
    fresh = _sim(pos, ori, precision="mixed_bf16")
    with pytest.raises(C.RigidFibersError) as e:
        solve_packed([fresh])
    assert e.value.status == C.RF_E_STATE
    m10 = _sim(pos, ori, precision="mixed_bf16", refinement_restart=10)
    m20 = _sim(pos, ori, precision="mixed_bf16", refinement_restart=20)
    m10.assembleSystem()
    m20.assembleSystem()
    with pytest.raises(C.RigidFibersError) as e:
        solve_packed([m10, m20])
    assert e.value.status == C.RF_E_INPUT


def test_server_pack_result_alone_equals_result_in_the_mix():
    from rigidfibers_b200 import Config
    from rigidfibers_b200.server import Server
    small = _layout(24, 11)
    cfg = Config(precision="mixed_bf16")
    with Server(max_active=4, pack_max_fibers=64) as srv:
        rid = srv.submit(cfg, *small, nsteps=4)
        srv.drain(timeout=300)
        ref = srv.result(rid)
    with Server(max_active=4, pack_max_fibers=64) as srv:
        ids = [srv.submit(Config(precision="mixed_bf16", slenderness=0.005), *_layout(50, 12), nsteps=6),
               srv.submit(cfg, *small, nsteps=4),
               srv.submit(Config(precision="mixed_bf16"), *_layout(300, 13), nsteps=3),   # its own handle
               srv.submit(cfg, *_layout(9, 14), nsteps=2)]
        srv.drain(timeout=300)
        assert [srv.poll(i)[0] for i in ids] == ["done"] * 4
        got = srv.result(ids[1])
        st = srv.stats()
    for a, b in zip(ref[:4], got[:4]):
        assert np.array_equal(a, b)
    assert got[4]["steps_done"] == 4
    assert st["completed"] == 4 and st["steps"] == 6 + 4 + 3 + 2
