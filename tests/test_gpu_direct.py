"""Direct solver (--magma): blocked LU with partial pivoting + FP64-residual
refinement, against the reference's direct-solve golden files and LAPACK.

Bounds: golden fields within 1e-5 relative (the golden files are FP64 runs of
the reference's sgesv path); general matrices within 1e-5 of an FP64 LAPACK
solve after refinement to ||b - A x|| / ||b|| <= 1e-7.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = [("BVec", "b"), ("XVec", "x"), ("TRANSVel", "tvel"), ("ROTVel", "rvel"), ("POS", "pos"), ("ORIENT", "ori")]


def _rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("integ", ["numeric", "analytic"])
def test_golden_direct(golden, integ):
    from rigidfibers_b200 import Config, Simulation
    sim = Simulation(Config(solver="direct", integration="numerical" if integ == "numeric" else "analytical"),
                     golden["positions"], golden["orientations"])
    for t in range(2):
        sim.assembleSystem()
        _, b = sim.system(with_matrix=False)
        sim.solveSystem()
        x = sim.solution()
        sim.updateVelocities()
        tv, rv = sim.velocities()
        sim.updateFibers(t == 0)
        p, o = sim.state()
        got = dict(b=b, x=x, tvel=tv, rvel=rv, pos=p, ori=o)
        for f, k in FIELDS:
            ref = golden["%s_direct/%d_%s" % (integ, t, f)]
            assert _rel(got[k], ref) <= 1e-5, (t, f, _rel(got[k], ref))
        st = sim.stats()
        assert st["relative_residual"] <= 1e-6
        # the TF32 tensor-core factors alone suffice for these systems
        assert st["factorizations"] == 1 and st["refinement_steps"] <= 4 and st["pivoted"] == 0


def _lu_solve(A, b, tol=1e-7):
    import torch
    from rigidfibers_b200 import _capi as C
    R = A.shape[0]
    Ad = torch.from_numpy(np.asfortranarray(A, np.float32).reshape(-1, order="F").copy()).cuda()
    bd = torch.from_numpy(np.asarray(b, np.float32)).cuda()
    xd = torch.zeros(R, device="cuda")
    rc = C.load().rf_dense_lu_solve(ctypes.c_void_p(Ad.data_ptr()), ctypes.c_void_p(bd.data_ptr()),
                                    ctypes.c_void_p(xd.data_ptr()), R, tol,
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, xd.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("R", [1, 5, 64, 100, 131, 300])
def test_lu_random_matrix_needs_pivoting(R):
    rng = np.random.default_rng(R)
    A = rng.standard_normal((R, R)).astype(np.float32)
    b = rng.standard_normal(R).astype(np.float32)
    rc, x = _lu_solve(A, b)
    assert rc == 0
    ref = np.linalg.solve(A.astype(np.float64), b.astype(np.float64))
    assert _rel(x, ref) <= 1e-5


def test_lu_permutation_matrix():
    R = 130
    rng = np.random.default_rng(1)
    P = np.eye(R, dtype=np.float32)[rng.permutation(R)]
    b = rng.standard_normal(R).astype(np.float32)
    rc, x = _lu_solve(P, b)
    assert rc == 0
    assert np.abs(x - np.linalg.solve(P.astype(np.float64), b)).max() < 1e-6


def test_lu_singular_matrix_reports_error():
    from rigidfibers_b200 import _capi as C
    R = 70
    rng = np.random.default_rng(2)
    A = rng.standard_normal((R, R)).astype(np.float32)
    A[:, 33] = 0.0
    rc, _ = _lu_solve(A, np.ones(R, np.float32))
    assert rc == C.RF_E_SINGULAR


@pytest.mark.parametrize("R", [1, 37, 128, 131, 256, 300, 640, 1000, 4099])
def test_lu_without_row_exchanges_on_dominant_matrices(R):
    """Matrices of this problem's kind (identity plus small couplings): every
    multiplier of the unpivoted factorization is below 1, so partial pivoting
    would exchange no row and the tensor-core factorization is kept (sizes
    cover partial last panels, a single panel, and panel pairs); within 1e-5 of
    an FP64 LAPACK solve after refinement."""
    rng = np.random.default_rng(100 + R)
    A = (np.eye(R) + 0.4 * rng.standard_normal((R, R)) / np.sqrt(R)).astype(np.float32)
    b = rng.standard_normal(R).astype(np.float32)
    rc, x = _lu_solve(A, b)
    assert rc == 0
    ref = np.linalg.solve(A.astype(np.float64), b.astype(np.float64))
    assert _rel(x, ref) <= 1e-5


def test_fiber_system_is_factored_without_row_exchanges():
    """An N=300 suspension at the precision configuration's density: the
    direct solver keeps the exchange-free tensor-core factors (stats.pivoted 0)
    and its forces match the FP64 oracle within 1e-5."""
    from oracle import oracle as O
    from rigidfibers_b200 import Config, Simulation
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    n = 300
    pos, ori = sphere_layout(n, 18.0 * (n / 4000.0) ** (1 / 3), 0.2, seed=layout_seed(3, n))
    sim = Simulation(Config(solver="direct"), pos, ori)
    sim.assembleSystem()
    sim.solveSystem()
    st = sim.stats()
    assert st["pivoted"] == 0 and st["relative_residual"] <= 1e-6
    A64, b64 = O.assemble(pos, ori, O.Params(), False, np.float64)
    ref = np.linalg.solve(A64, b64)
    assert _rel(sim.solution(), ref) <= 1e-5


def test_random_matrix_falls_back_to_row_exchanges():
    """A general random matrix has multipliers above 1, so the exchange-free
    factors are discarded and the matrix is factored again with partial
    pivoting (through the standalone entry point); the answer matches LAPACK."""
    rng = np.random.default_rng(7)
    R = 700
    A = rng.standard_normal((R, R)).astype(np.float32)
    b = rng.standard_normal(R).astype(np.float32)
    rc, x = _lu_solve(A, b)
    assert rc == 0
    assert _rel(x, np.linalg.solve(A.astype(np.float64), b.astype(np.float64))) <= 1e-5


@pytest.mark.parametrize("big", [5.0, 300.0])
def test_static_pivoting_and_its_fallback(big):
    """Multipliers above 1 (a row exchange under partial pivoting): with the
    largest at 5 the factors without exchanges are kept (static pivoting) and
    the FP64 refinement recovers the accuracy; at 300 they exceed the limit of
    64 and the matrix is refactored with partial pivoting.  Either way the
    solution matches LAPACK within 1e-5."""
    rng = np.random.default_rng(int(big))
    R = 700
    A = np.eye(R) + 0.2 * rng.standard_normal((R, R)) / np.sqrt(R)
    for i, j in ((3, 200), (150, 400), (500, 650)):
        A[j, i] = big                     # row j, column i: l_ji ~ big
    A = A.astype(np.float32)
    b = rng.standard_normal(R).astype(np.float32)
    rc, x = _lu_solve(A, b)
    assert rc == 0
    assert _rel(x, np.linalg.solve(A.astype(np.float64), b.astype(np.float64))) <= 1e-5


def test_evolving_suspension_direct_steps_match_fp64():
    """Three direct-solver steps of an N=400 suspension at the precision
    configuration's density (nearly touching pairs appear as it evolves): the
    forces stay within 1e-5 of the FP64 oracle's solve of the same FP32-formed
    system, whichever factorization was kept."""
    from oracle import oracle as O
    from rigidfibers_b200 import Config, Simulation
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    n = 400
    pos, ori = sphere_layout(n, 18.0 * (n / 4000.0) ** (1 / 3), 0.2, seed=layout_seed(3, n))
    sim = Simulation(Config(solver="direct"), pos, ori)
    for t in range(3):
        p0, o0 = sim.state()
        sim.assembleSystem()
        sim.solveSystem()
        st = sim.stats()
        assert st["relative_residual"] <= 1e-6
        assert st["max_multiplier"] > 0.0
        A64, b64 = O.assemble(p0, o0, O.Params(), False, np.float64)
        assert _rel(sim.solution(), np.linalg.solve(A64, b64)) <= 1e-5
        sim.updateVelocities()
        sim.updateFibers(t == 0)
