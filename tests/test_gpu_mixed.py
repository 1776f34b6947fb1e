"""Mixed-precision path: structured operator (FP32 + 16-bit pair blocks),
GMRES with FP64-residual refinement, velocities from the stored blocks.

Bounds (written here): forces, velocities and fiber
state within 1e-4 relative of the FP64 oracle; the structured FP32 operator
within twice the REAL*4 oracle's own error; the 16-bit operators within
their storage precision (FP16 2e-3, BF16 1.5e-2 of the largest |y|).
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


@pytest.mark.parametrize("n", [1, 2, 5, 16, 17, 40, 100])
@pytest.mark.parametrize("prec", ["mixed_fp16", "mixed_bf16"])
def test_structured_operator_matches_dense(n, prec):
    pos, ori = sphere_layout(n, radius=max(1.5, 0.8 * n ** (1 / 3)), seed=21 + n)
    sim = _sim(pos, ori, precision=prec)
    sim.assembleSystem()
    p = O.Params()
    A64, b64 = O.assemble(pos, ori, p, False, np.float64)
    A32, b32 = O.assemble(pos, ori, p, False, np.float32)
    rng = np.random.default_rng(n)
    x = rng.standard_normal(15 * n)
    yref = A64 @ x
    y32ref = A32.astype(np.float64) @ x
    y = sim.apply_operator(x, 0)
    assert _rel(y, yref) <= max(2e-6, 2 * _rel(y32ref, yref))
    y16 = sim.apply_operator(x, 1)
    assert _rel(y16, yref) <= (2e-3 if prec == "mixed_fp16" else 1.5e-2)
    _, b = sim.system(with_matrix=False)
    if n > 1:
        assert _rel(b, b64) <= max(2e-6, 2 * _rel(b32, b64))


@pytest.mark.parametrize("m", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("n", [17, 40])
def test_structured_operator_other_force_terms(m, n):
    """The TMA-staged kernels split a pair's M^2 blocks between two threads at
    a 16-byte boundary of its record (M <= 5); M > 5 uses the register-staged
    kernels.  Same bounds as the M = 5 test."""
    pos, ori = sphere_layout(n, radius=max(1.5, 0.8 * n ** (1 / 3)), seed=31 + n + m)
    sim = _sim(pos, ori, precision="mixed_fp16", number_of_terms_in_force_expansion=m)
    sim.assembleSystem()
    p = O.Params(M=m)
    A64, _ = O.assemble(pos, ori, p, False, np.float64)
    A32, _ = O.assemble(pos, ori, p, False, np.float32)
    x = np.random.default_rng(n + m).standard_normal(3 * m * n)
    yref = A64 @ x
    y32ref = A32.astype(np.float64) @ x
    assert _rel(sim.apply_operator(x, 0), yref) <= max(2e-6, 2 * _rel(y32ref, yref))
    assert _rel(sim.apply_operator(x, 1), yref) <= 2e-3


def _run(sim, nsteps):
    out = []
    for t in range(nsteps):
        sim.assembleSystem()
        sim.solveSystem()
        x = sim.solution()
        sim.updateVelocities()
        tv, rv = sim.velocities()
        sim.updateFibers(t == 0)
        pos, ori = sim.state()
        out.append(dict(x=x, tvel=tv, rvel=rv, pos=pos, ori=ori, stats=sim.stats()))
    return out


@pytest.mark.parametrize("prec", ["mixed_fp16", "mixed_bf16"])
def test_mixed_steps_within_1e4_of_fp64(prec):
    pos, ori = sphere_layout(200, radius=4.0, seed=7)
    ref = O.run_steps(pos, ori, O.Params(), 3, solver="direct", dtype=np.float64)
    res = _run(_sim(pos, ori, precision=prec, refinement_tolerance=1e-6), 3)
    for t in range(3):
        for k in ("x", "tvel", "rvel", "pos", "ori"):
            assert _rel(res[t][k], ref[t][k]) <= 1e-4, (prec, t, k, _rel(res[t][k], ref[t][k]))
        st = res[t]["stats"]
        assert st["relative_residual"] <= 1e-6
        assert st["refinement_steps"] >= 1


@pytest.mark.parametrize("prec", ["mixed_fp16", "mixed_bf16"])
def test_mixed_bicgstab_steps_within_1e4_of_fp64(prec):
    """BiCGSTAB on the 16-bit pair blocks (FP32 sums) inside FP64-residual
    refinement (the reference's BiCGSTAB call: src/simulation.cu:424-427):
    forces, velocities and fiber state within 1e-4 of the FP64 oracle over
    three steps, the FP64 residual at the refinement target."""
    pos, ori = sphere_layout(200, radius=4.0, seed=7)
    ref = O.run_steps(pos, ori, O.Params(), 3, solver="direct", dtype=np.float64)
    res = _run(_sim(pos, ori, precision=prec, solver="bicgstab", refinement_tolerance=1e-6), 3)
    for t in range(3):
        for k in ("x", "tvel", "rvel", "pos", "ori"):
            assert _rel(res[t][k], ref[t][k]) <= 1e-4, (prec, t, k, _rel(res[t][k], ref[t][k]))
        st = res[t]["stats"]
        assert st["relative_residual"] <= 1e-6
        assert st["refinement_steps"] >= 1 and st["iterations"] > 0


def test_mixed_bicgstab_matches_mixed_gmres():
    """Both refined solves reach ||b - A x|| / ||b|| <= 1e-6 on the same FP32
    blocks, so their forces agree far inside the 1e-4 bound."""
    pos, ori = sphere_layout(120, radius=3.5, seed=17)
    a = _run(_sim(pos, ori, precision="mixed_fp16", solver="bicgstab"), 2)
    b = _run(_sim(pos, ori, precision="mixed_fp16"), 2)
    for t in range(2):
        for k in ("x", "tvel", "rvel", "pos"):
            assert _rel(a[t][k], b[t][k]) <= 1e-5, (t, k, _rel(a[t][k], b[t][k]))


def test_mixed_rejects_direct_solver():
    from rigidfibers_b200 import RigidFibersError
    from rigidfibers_b200 import _capi as C
    pos, ori = sphere_layout(4, radius=1.5, seed=1)
    with pytest.raises(RigidFibersError) as e:
        _sim(pos, ori, precision="mixed_fp16", solver="direct")
    assert e.value.status == C.RF_E_UNSUPPORTED


def test_mixed_golden(golden):
    """The reference's golden files (FP64 runs) through the mixed path."""
    res = _run(_sim(golden["positions"], golden["orientations"], precision="mixed_fp16"), 2)
    for t in range(2):
        for f, k in [("XVec", "x"), ("TRANSVel", "tvel"), ("ROTVel", "rvel"), ("POS", "pos"), ("ORIENT", "ori")]:
            ref = golden["numeric_direct/%d_%s" % (t, f)]
            assert _rel(res[t][k], ref) <= 1e-4, (t, f)


def test_mixed_and_fp32_agree():
    pos, ori = sphere_layout(150, radius=3.5, seed=8)
    a = _run(_sim(pos, ori, precision="mixed_fp16"), 2)
    b = _run(_sim(pos, ori, gmres_tolerance=2e-6), 2)   # near the FP32 residual floor
    for t in range(2):
        for k in ("x", "tvel", "rvel", "pos"):
            assert _rel(a[t][k], b[t][k]) <= 1e-4, (t, k)


def test_mixed_requires_numerical_integration():
    from rigidfibers_b200 import RigidFibersError
    from rigidfibers_b200 import _capi as C
    pos, ori = sphere_layout(4, radius=1.5, seed=1)
    with pytest.raises(RigidFibersError) as e:
        _sim(pos, ori, precision="mixed_fp16", integration="analytical")
    assert e.value.status == C.RF_E_UNSUPPORTED


@pytest.mark.parametrize("prec", ["fp32", "mixed_fp16"])
def test_autotune_keeps_the_solution(prec):
    """rf_autotune times the matvec launch choices and keeps the fastest; the
    solution stays within 1e-5 of the untuned one (only the summation order of
    the matvec changes) and a second call is served from the cache."""
    from rigidfibers_b200 import Config, Simulation
    pos, ori = sphere_layout(80, 4.0, seed=31)
    ref = Simulation(Config(precision=prec), pos, ori)
    ref.run(2)
    p0, o0 = ref.state()
    ref.close()
    sim = Simulation(Config(precision=prec), pos, ori)
    rep = sim.autotune()
    if prec == "fp32":
        assert rep["gemv_ctas_per_sm"] in (2, 4, 8, 16)
        assert min(v for v in rep["gemv_ms"] if v > 0) > 0
    else:
        assert rep["matvec_variant"] in (0, 2) and min(rep["matvec_ms"]) > 0
    assert rep["asm_variant"] in (0, 1) and min(rep["asm_ms"]) > 0
    sim.run(2)
    p1, o1 = sim.state()
    assert _rel(p1, p0) <= 1e-5 and _rel(o1, o0) <= 1e-5
    again = Simulation(Config(precision=prec), pos, ori)
    assert again.autotune()["cached"]


@pytest.mark.parametrize("n", [7, 40, 130])
@pytest.mark.parametrize("prec", ["fp32", "mixed_fp16", "mixed_bf16"])
def test_assembly_variants_are_bit_identical(n, prec):
    """The numerical pair-tile kernels (scalar FP32 and packed two-lane FP32)
    round every step the same way: the dense operator and right-hand side are
    equal bit for bit, and so are two whole steps of the structured path."""
    from rigidfibers_b200 import _capi as C
    pos, ori = sphere_layout(n, radius=max(1.5, 0.8 * n ** (1 / 3)), seed=41 + n)
    out = []
    for v in (0, 1):
        sim = _sim(pos, ori, precision=prec)
        C.check(C.load().rf_set_assembly_variant(sim._h, v), "rf_set_assembly_variant")
        sim.assembleSystem()
        A, b = sim.system(with_matrix=prec == "fp32")
        sim.run(2)
        p, o = sim.state()
        out.append((A, b, p, o))
        sim.close()
    for a, b in zip(out[0], out[1]):
        if a is not None:
            assert np.array_equal(np.asarray(a), np.asarray(b))
    with pytest.raises(Exception):
        sim = _sim(pos, ori, precision=prec)
        try:
            C.check(C.load().rf_set_assembly_variant(sim._h, 2), "rf_set_assembly_variant")
        finally:
            sim.close()
