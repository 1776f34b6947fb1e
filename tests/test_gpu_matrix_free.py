"""Matrix-free mode (RF_PREC_MATRIX_FREE): no operator stored, every Krylov
product recomputes the pair blocks and applies them to the vector.

Bounds (written here): the product within 2e-6 of the largest |y| of the
dense FP32 operator's product (same blocks, another summation order); the
right-hand side within 1e-6 relative of the dense path's; three steps within
1e-5 of the FP64 oracle (GMRES tolerance 1e-7), the plain path's bound.
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


@pytest.mark.parametrize("n", [1, 2, 7, 9, 40, 130])
def test_matrix_free_product_equals_the_dense_operator(n):
    pos, ori = sphere_layout(n, radius=max(1.5, 0.8 * n ** (1 / 3)), seed=61 + n)
    dense = _sim(pos, ori, precision="fp32")
    free = _sim(pos, ori, precision="matrix_free")
    dense.assembleSystem()
    free.assembleSystem()
    _, bd = dense.system(with_matrix=False)
    _, bf = free.system(with_matrix=False)
    assert _rel(bf, bd) <= 1e-6
    rng = np.random.default_rng(n)
    for _ in range(2):   # twice: every partial row is rewritten by each product
        x = rng.standard_normal(15 * n)
        yd = dense.apply_operator(x)
        yf = free.apply_operator(x)
        assert np.abs(yf - yd).max() <= 2e-6 * np.abs(yd).max()


@pytest.mark.parametrize("solver", ["gmres", "bicgstab"])
def test_matrix_free_steps_match_fp64_oracle(solver):
    pos, ori = sphere_layout(37, radius=2.5, seed=5)
    ref = O.run_steps(pos, ori, O.Params(), 3, solver="direct", dtype=np.float64)
    kw = {"gmres_tolerance": 1e-7} if solver == "gmres" else {"bicgstab_tolerance": 1e-7}
    sim = _sim(pos, ori, precision="matrix_free", solver=solver, **kw)
    for t in range(3):
        sim.step(t)
        p, o = sim.state()
        tv, rv = sim.velocities()
        x = sim.solution()
        for got, k in ((x, "x"), (tv, "tvel"), (rv, "rvel"), (p, "pos"), (o, "ori")):
            assert _rel(got, ref[t][k]) <= 1e-5, (t, k, _rel(got, ref[t][k]))


def test_matrix_free_gmres_iterations_match_the_dense_path():
    pos, ori = sphere_layout(150, radius=4.5, seed=17)
    its = {}
    for prec in ("fp32", "matrix_free"):
        sim = _sim(pos, ori, precision=prec)
        its[prec] = []
        for t in range(2):
            sim.step(t)
            its[prec].append(sim.stats()["iterations"])
        sim.close()
    assert all(abs(a - b) <= 1 for a, b in zip(its["fp32"], its["matrix_free"])), its


def test_matrix_free_has_no_matrix_to_read():
    from rigidfibers_b200 import RigidFibersError
    pos, ori = sphere_layout(5, radius=1.5, seed=3)
    sim = _sim(pos, ori, precision="matrix_free")
    sim.assembleSystem()
    with pytest.raises(RigidFibersError):
        sim.system(with_matrix=True)
    with pytest.raises(RigidFibersError):
        sim.apply_operator(np.ones(75), which=1)
