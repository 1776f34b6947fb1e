"""ctypes front end of the CPU oracle (oracle/rf_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference arm, as the checker.  The product
(rigidfibers_b200) never imports it.

`run_steps` follows the time loop of the reference's Fortran program
(fortran/fibers.f95:182-349): assemble -> solve -> update velocities ->
update fibers, then rotate previous/current/next buffers.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librf_oracle.so")
_lib = None


def build():
    """Compile the oracle with its Makefile (system g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        for suf in ("f32", "f64"):
            for name in ("assemble", "assemble_rows", "update_velocities", "gmres", "bicgstab",
                         "lu_solve", "gemv", "update_fibers", "tables"):
                getattr(_lib, "rfo_%s_%s" % (name, suf)).restype = ctypes.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _suf(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


class Params:
    """Simulation parameters with the reference's .ini meaning
    (tests/config.ini:18-37)."""

    def __init__(self, M=5, intervals=8, eps=0.01, dt=0.1, restart=10, maxit=1000, tol=1e-5,
                 bicgstab_maxit=1000, bicgstab_tol=1e-5):
        self.M, self.intervals, self.eps, self.dt = M, intervals, eps, dt
        self.restart, self.maxit, self.tol = restart, maxit, tol
        self.bicgstab_maxit, self.bicgstab_tol = bicgstab_maxit, bicgstab_tol


def tables(p, dtype=np.float64):
    dt = np.dtype(dtype)
    Q = 3 * p.intervals
    pts, wts = np.zeros(Q, dt), np.zeros(Q, dt)
    leg = np.zeros(Q * p.M, dt)
    lam, eig = np.zeros(p.M, dt), np.zeros(p.M, dt)
    getattr(lib(), "rfo_tables_" + _suf(dt))(p.M, p.intervals, ctypes.c_double(p.eps), _p(pts), _p(wts),
                                              _p(leg), _p(lam), _p(eig))
    return pts, wts, leg.reshape(Q, p.M), lam, eig


def assemble(pos, ori, p, analytical=False, dtype=np.float32):
    """Returns (A, b); A is an (R, R) Fortran-ordered (column-major) array."""
    dt = np.dtype(dtype)
    pos = np.ascontiguousarray(pos, dt).reshape(-1)
    ori = np.ascontiguousarray(ori, dt).reshape(-1)
    N = pos.size // 3
    R = 3 * p.M * N
    A = np.zeros((R, R), dt, order="F")
    b = np.zeros(R, dt)
    getattr(lib(), "rfo_assemble_" + _suf(dt))(N, p.M, p.intervals, ctypes.c_double(p.eps), int(analytical),
                                                _p(pos), _p(ori), _p(A), _p(b))
    return A, b


def assemble_rows(pos, ori, p, i0, i1, analytical=False, dtype=np.float32):
    """Row slab of fibers [i0, i1): ((i1-i0)*3M, R) Fortran-ordered, and b rows."""
    dt = np.dtype(dtype)
    pos = np.ascontiguousarray(pos, dt).reshape(-1)
    ori = np.ascontiguousarray(ori, dt).reshape(-1)
    N = pos.size // 3
    R = 3 * p.M * N
    rows = (i1 - i0) * 3 * p.M
    slab = np.zeros((rows, R), dt, order="F")
    b = np.zeros(rows, dt)
    getattr(lib(), "rfo_assemble_rows_" + _suf(dt))(N, p.M, p.intervals, ctypes.c_double(p.eps),
                                                     int(analytical), _p(pos), _p(ori), i0, i1, _p(slab), _p(b))
    return slab, b


def update_velocities(pos, ori, coeff, p, i0=0, i1=None, dtype=np.float32, analytical=False):
    """Translational and rotational velocities (fortran/update_velocities.incl).
    analytical=True integrates the inner integral in closed form, which is
    what the reference's 100_analytic_* golden files were produced with; the
    committed Fortran/CUDA code always integrates numerically."""
    dt = np.dtype(dtype)
    pos = np.ascontiguousarray(pos, dt).reshape(-1)
    ori = np.ascontiguousarray(ori, dt).reshape(-1)
    coeff = np.ascontiguousarray(coeff, dt).reshape(-1)
    N = pos.size // 3
    i1 = N if i1 is None else i1
    tv = np.zeros(3 * N, dt)
    rv = np.zeros(3 * N, dt)
    getattr(lib(), "rfo_update_velocities_" + _suf(dt))(N, p.M, p.intervals, ctypes.c_double(p.eps), _p(pos),
                                                         _p(ori), _p(coeff), i0, i1, _p(tv), _p(rv),
                                                         int(analytical))
    return tv.reshape(N, 3), rv.reshape(N, 3)


def gemv(A, x):
    A = np.asfortranarray(A)
    x = np.ascontiguousarray(x, A.dtype)
    y = np.zeros(A.shape[0], A.dtype)
    getattr(lib(), "rfo_gemv_" + _suf(A.dtype))(A.shape[0], A.shape[1], _p(A), _p(x), _p(y))
    return y


def solve(A, b, p, solver="gmres"):
    """Returns (x, iterations, relative residual).  A is not modified."""
    dt = A.dtype
    n = A.shape[0]
    A = np.asfortranarray(A)
    b = np.ascontiguousarray(b, dt)
    rel = ctypes.c_double(0.0)
    if solver == "gmres":
        x = np.zeros(n, dt)
        it = getattr(lib(), "rfo_gmres_" + _suf(dt))(n, _p(A), _p(b), _p(x), p.restart, p.maxit,
                                                     ctypes.c_double(p.tol), ctypes.byref(rel))
        return x, it, rel.value
    if solver == "bicgstab":
        x = np.zeros(n, dt)
        it = getattr(lib(), "rfo_bicgstab_" + _suf(dt))(n, _p(A), _p(b), _p(x), p.bicgstab_maxit,
                                                        ctypes.c_double(p.bicgstab_tol), 200, ctypes.byref(rel))
        return x, it, rel.value
    if solver == "direct":
        LU = np.array(A, order="F", copy=True)
        x = b.copy()
        info = getattr(lib(), "rfo_lu_solve_" + _suf(dt))(n, _p(LU), _p(x))
        if info != 0:
            raise RuntimeError("singular matrix at column %d" % info)
        return x, 0, float(np.linalg.norm(gemv(A, x) - b) / np.linalg.norm(b))
    raise ValueError(solver)


def update_fibers(first, dt_, prev_pos, cur_pos, prev_ori, cur_ori, prev_tv, cur_tv, prev_rv, cur_rv):
    dt = cur_pos.dtype
    arrs = [np.ascontiguousarray(a, dt).reshape(-1) for a in
            (prev_pos, cur_pos, prev_ori, cur_ori, prev_tv, cur_tv, prev_rv, cur_rv)]
    N = arrs[1].size // 3
    npos = np.zeros(3 * N, dt)
    nori = np.zeros(3 * N, dt)
    getattr(lib(), "rfo_update_fibers_" + _suf(dt))(N, int(first), ctypes.c_double(dt_), *[_p(a) for a in arrs],
                                                     _p(npos), _p(nori))
    return npos.reshape(N, 3), nori.reshape(N, 3)


def run_steps(pos0, ori0, p, nsteps, analytical=False, solver="gmres", dtype=np.float32, keep_A=False,
              analytical_velocities=None):
    """The reference time loop (fortran/fibers.f95:182-349).  Returns one dict
    per step with the validate-mode dumps: b (BVec), x (XVec), tvel, rvel,
    next positions / orientations, and the solver's iteration count."""
    dt = np.dtype(dtype)
    cur_pos = np.array(pos0, dt).reshape(-1, 3)
    cur_ori = np.array(ori0, dt).reshape(-1, 3)
    prev_pos = cur_pos.copy()
    prev_ori = cur_ori.copy()
    prev_tv = np.zeros_like(cur_pos)
    prev_rv = np.zeros_like(cur_pos)
    out = []
    for t in range(nsteps):
        A, b = assemble(cur_pos, cur_ori, p, analytical, dt)
        x, it, rel = solve(A, b, p, solver)
        av = analytical if analytical_velocities is None else analytical_velocities
        tv, rv = update_velocities(cur_pos, cur_ori, x, p, dtype=dt, analytical=av)
        npos, nori = update_fibers(t == 0, p.dt, prev_pos, cur_pos, prev_ori, cur_ori, prev_tv, tv, prev_rv, rv)
        rec = dict(b=b, x=x, tvel=tv, rvel=rv, pos=npos, ori=nori, iterations=it, relres=rel)
        if keep_A:
            rec["A"] = A
        out.append(rec)
        prev_pos, cur_pos = cur_pos, npos
        prev_ori, cur_ori = cur_ori, nori
        prev_tv, prev_rv = tv, rv
    return out
