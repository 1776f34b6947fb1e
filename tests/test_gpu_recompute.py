"""Recompute modes (RF_PREC_MIXED_*_RECOMPUTE): the mixed-precision solve with
only the 16-bit pair records stored; the FP64 refinement residual and the
velocities form the FP32 blocks again from the fibers.

Bounds (written here): the solution, velocities and state within 1e-5
relative of the mixed mode that stores the FP32 blocks (the same 16-bit
operator inside the Krylov solve; the residual's products differ in summation
order); three steps within 1e-4 of the FP64 oracle, the mixed modes' bound.
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


@pytest.mark.parametrize("p16", ["fp16", "bf16"])
@pytest.mark.parametrize("solver", ["gmres", "bicgstab"])
def test_recompute_follows_the_stored_mixed_mode(p16, solver):
    pos, ori = sphere_layout(120, radius=4.0, seed=23)
    full = _sim(pos, ori, precision="mixed_" + p16, solver=solver)
    lean = _sim(pos, ori, precision="mixed_%s_recompute" % p16, solver=solver)
    assert lean.stats()["device_bytes"] < 0.5 * full.stats()["device_bytes"]
    for t in range(2):
        full.step(t)
        lean.step(t)
        st = lean.stats()
        assert st["relative_residual"] <= 1e-6 and st["refinement_steps"] >= 1
        assert _rel(lean.solution(), full.solution()) <= 1e-5, t
        for a, b in zip(lean.velocities(), full.velocities()):
            assert _rel(a, b) <= 1e-5, t
        for a, b in zip(lean.state(), full.state()):
            assert _rel(a, b) <= 1e-5, t
    full.close()
    lean.close()


def test_recompute_steps_within_1e4_of_fp64():
    pos, ori = sphere_layout(60, radius=3.0, seed=29)
    ref = O.run_steps(pos, ori, O.Params(), 3, solver="direct", dtype=np.float64)
    sim = _sim(pos, ori, precision="mixed_fp16_recompute")
    for t in range(3):
        sim.step(t)
        p, o = sim.state()
        tv, rv = sim.velocities()
        for got, k in ((sim.solution(), "x"), (tv, "tvel"), (rv, "rvel"), (p, "pos"), (o, "ori")):
            assert _rel(got, ref[t][k]) <= 1e-4, (t, k, _rel(got, ref[t][k]))
    sim.close()


def test_recompute_operator_products():
    """apply_operator(which=0) forms the FP32 blocks again (the matrix-free
    product), which=1 reads the stored 16-bit records: both as in the mixed
    mode that stores the FP32 copy."""
    pos, ori = sphere_layout(40, radius=2.5, seed=31)
    full = _sim(pos, ori, precision="mixed_bf16")
    lean = _sim(pos, ori, precision="mixed_bf16_recompute")
    full.assembleSystem()
    lean.assembleSystem()
    _, bf = full.system(with_matrix=False)
    _, bl = lean.system(with_matrix=False)
    assert np.array_equal(bf, bl)
    x = np.random.default_rng(2).standard_normal(15 * 40)
    y32, y16 = full.apply_operator(x), full.apply_operator(x, which=1)
    assert np.abs(lean.apply_operator(x) - y32).max() <= 2e-6 * np.abs(y32).max()
    assert np.array_equal(lean.apply_operator(x, which=1), y16)
    full.close()
    lean.close()
