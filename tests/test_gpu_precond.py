"""Near-field preconditioner (rf_set_near_field_preconditioner): each fiber's
rows of the inverse of its neighbourhood block, applied on the right inside
flexible GMRES-IR.

Bounds (written here): on the same system the solution, velocities and new
state within 1e-5 relative of the unpreconditioned solve (both converge to
the same FP64 residual tolerance, 1e-6); three steps within 1e-4 of the FP64
oracle;
fewer GMRES iterations than without it; whole-step graphs bit-identical to
direct launches.
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


def _sim(pos, ori, **kw):
    from rigidfibers_b200 import Config, Simulation
    return Simulation(Config(**kw), pos, ori)


def _layout(n, seed):
    # the N=4000 benchmark's density: 4000 fibers in a sphere of radius 18
    return sphere_layout(n, 18.0 * (n / 4000.0) ** (1.0 / 3.0), 0.2, seed=seed)


@pytest.mark.parametrize("k", [1, 4, 8])
def test_preconditioned_solve_follows_the_plain_one(k):
    pos, ori = _layout(400, 3)
    plain = _sim(pos, ori, precision="mixed_fp16")
    pre = _sim(pos, ori, precision="mixed_fp16")
    pre.set_near_field_preconditioner(k)
    its = [[], []]
    for t in range(3):
        plain.step(t)
        pre.step(t)
        its[0].append(plain.stats()["iterations"])
        its[1].append(pre.stats()["iterations"])
        assert pre.stats()["relative_residual"] <= 1e-6
        if t == 0:   # the same system (later steps start from states that differ by ~1e-5)
            assert _rel(pre.solution(), plain.solution()) <= 1e-5
            for a, b in zip(pre.velocities(), plain.velocities()):
                assert _rel(a, b) <= 1e-5
            for a, b in zip(pre.state(), plain.state()):
                assert _rel(a, b) <= 1e-5
    if k >= 4:
        assert sum(its[1]) < 0.75 * sum(its[0]), its
    plain.close()
    pre.close()


def test_preconditioned_steps_within_1e4_of_fp64():
    pos, ori = _layout(60, 5)
    ref = O.run_steps(pos, ori, O.Params(), 3, solver="direct", dtype=np.float64)
    sim = _sim(pos, ori, precision="mixed_bf16")
    sim.set_near_field_preconditioner(4)
    for t in range(3):
        sim.step(t)
        p, o = sim.state()
        tv, rv = sim.velocities()
        for got, key in ((sim.solution(), "x"), (tv, "tvel"), (rv, "rvel"), (p, "pos"), (o, "ori")):
            assert _rel(got, ref[t][key]) <= 1e-4, (t, key)
    sim.close()


def test_preconditioned_graphs_equal_direct_launches():
    pos, ori = _layout(200, 9)
    out = []
    for mode in (0, 1, 2):
        sim = _sim(pos, ori, precision="mixed_fp16")
        sim.set_near_field_preconditioner(4)
        sim.set_cuda_graphs(mode)
        for t in range(3):
            sim.step(t)
        out.append(sim.state() + sim.velocities())
        sim.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert np.array_equal(a, b)


def test_preconditioner_refusals():
    from rigidfibers_b200 import _capi as C
    pos, ori = _layout(20, 11)
    for kw in (dict(precision="fp32"), dict(precision="matrix_free"), dict(precision="mixed_fp16_recompute"),
               dict(precision="mixed_fp16", solver="bicgstab")):
        sim = _sim(pos, ori, **kw)
        with pytest.raises(C.RigidFibersError) as e:
            sim.set_near_field_preconditioner(4)
        assert e.value.status == C.RF_E_UNSUPPORTED
        sim.set_near_field_preconditioner(0)
        sim.close()
    sim = _sim(pos, ori, precision="mixed_fp16")
    for bad in (-1, 9):
        with pytest.raises(C.RigidFibersError) as e:
            sim.set_near_field_preconditioner(bad)
        assert e.value.status == C.RF_E_INPUT
    sim.close()
