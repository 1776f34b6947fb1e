"""The CPU oracle against the reference's golden vectors.

The golden files (tests/reference/100_*/{0,1}_*.ref in the reference project,
packed by tests/golden/make_golden.py) hold F16.8 values, i.e. 5e-9
resolution.  They were produced in double precision: the FP64 oracle
reproduces every direct-solve field of both steps to that resolution.  The
REAL*4 oracle reproduces the numerical-integration fields to the FP32
tolerances written below.  The analytic golden files were produced with the
velocities integrated analytically as well (the committed
fortran/update_velocities.incl integrates numerically), which the
`analytical_velocities` option of the oracle reproduces.
"""
import numpy as np
import pytest

from oracle import oracle as O

FIELDS = [("BVec", "b"), ("XVec", "x"), ("TRANSVel", "tvel"), ("ROTVel", "rvel"), ("POS", "pos"),
          ("ORIENT", "ori")]
PRINT_RES = 6e-9  # F16.8 rounding (5e-9) plus a margin


def _err(rec, golden, var, t, f, k):
    return float(np.abs(np.asarray(rec[k], np.float64).reshape(-1) - golden["%s/%d_%s" % (var, t, f)]).max())


@pytest.mark.parametrize("var", ["numeric_direct", "analytic_direct"])
def test_fp64_oracle_reproduces_direct_goldens(golden, var):
    p = O.Params()
    res = O.run_steps(golden["positions"], golden["orientations"], p, 2, analytical=var.startswith("analytic"),
                      solver="direct", dtype=np.float64)
    for t in range(2):
        for f, k in FIELDS:
            assert _err(res[t], golden, var, t, f, k) <= PRINT_RES, (t, f)


@pytest.mark.parametrize("var", ["numeric_gmres", "analytic_gmres"])
def test_fp64_oracle_reproduces_gmres_goldens(golden, var):
    p = O.Params()
    res = O.run_steps(golden["positions"], golden["orientations"], p, 2, analytical=var.startswith("analytic"),
                      solver="gmres", dtype=np.float64)
    # step 0: same Krylov subspace, same iterate
    for f, k in FIELDS:
        assert _err(res[0], golden, var, 0, f, k) <= PRINT_RES, f
    # step 1: both runs stop inside the GMRES tolerance (1e-5 relative residual)
    assert _err(res[1], golden, var, 1, "BVec", "b") <= PRINT_RES
    assert _err(res[1], golden, var, 1, "XVec", "x") <= 2e-5
    assert _err(res[1], golden, var, 1, "TRANSVel", "tvel") <= 1e-5
    assert _err(res[1], golden, var, 1, "POS", "pos") <= 1e-6


@pytest.mark.parametrize("solver", ["gmres", "direct"])
def test_fp32_oracle_numeric_goldens(golden, solver):
    var = "numeric_" + solver
    p = O.Params()
    res = O.run_steps(golden["positions"], golden["orientations"], p, 2, analytical=False, solver=solver,
                      dtype=np.float32)
    tol = {"BVec": 1e-6, "XVec": 2e-5, "TRANSVel": 1e-5, "ROTVel": 5e-6, "POS": 2e-6, "ORIENT": 1e-6}
    for t in range(2):
        for f, k in FIELDS:
            assert _err(res[t], golden, var, t, f, k) <= tol[f], (t, f)


def test_committed_velocity_quirk_differs_from_analytic_goldens(golden):
    """With numerically integrated velocities (the committed reference code)
    the analytic golden velocities are off by ~1e-4: the analytic golden
    files were made with analytic velocities."""
    p = O.Params()
    res = O.run_steps(golden["positions"], golden["orientations"], p, 1, analytical=True, solver="direct",
                      dtype=np.float64, analytical_velocities=False)
    e = _err(res[0], golden, "analytic_direct", 0, "TRANSVel", "tvel")
    assert 1e-5 < e < 1e-3


def test_gmres_bicgstab_direct_agree():
    rng = np.random.default_rng(3)
    n = 300
    A = np.eye(n) + 0.02 * rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    p = O.Params(tol=1e-10, bicgstab_tol=1e-10)
    A = np.asfortranarray(A)
    xd, _, _ = O.solve(A, b, p, "direct")
    xg, itg, rg = O.solve(A, b, p, "gmres")
    xb, itb, rb = O.solve(A, b, p, "bicgstab")
    assert itg > 0 and itb > 0
    assert np.abs(xg - xd).max() < 1e-8
    assert np.abs(xb - xd).max() < 1e-8


def test_tables():
    p = O.Params()
    pts, wts, leg, lam, eig = O.tables(p)
    assert abs(wts.sum() - 2.0) < 1e-14
    assert np.allclose(pts, -pts[::-1])
    # P_1 = s, P_2 = (3s^2-1)/2
    assert np.allclose(leg[:, 0], pts)
    assert np.allclose(leg[:, 1], 0.5 * (3 * pts ** 2 - 1))
    # Gauss rule integrates P_k exactly to 0
    assert np.abs(wts @ leg).max() < 1e-14
    assert lam[0] == 2.0 and abs(lam[1] - 3.0) < 1e-15
