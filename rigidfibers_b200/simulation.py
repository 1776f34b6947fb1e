"""Host-side mirror of the reference's `Simulation` class
(src/simulation.h:38-97, src/simulation.cu:44-528) over the C ABI.

    sim = Simulation(config, positions, orientations)
    for t in range(config.number_of_timesteps):
        sim.step(t)                      # assembleSystem -> solveSystem ->
                                         # updateVelocities -> updateFibers

Every method raises RigidFibersError on a non-zero status; a solver that
hits its iteration limit raises unless `allow_noconv` is set (the reference
prints and continues, src/simulation.cu:441-442).
"""
import ctypes

import numpy as np

from . import _capi as C


class Config:
    """The reference's .ini keys plus the runtime choices it fixed at compile
    time (solver, integration) and the precision mode."""

    def __init__(self, **kw):
        lib = C.load()
        self._c = C.rf_config()
        C.check(lib.rf_config_default(ctypes.byref(self._c)), "rf_config_default")
        for k, v in kw.items():
            self[k] = v

    def __setitem__(self, key, value):
        if key == "solver":
            value = C.SOLVERS[value] if isinstance(value, str) else value
        elif key == "integration":
            value = C.INTEGRATIONS[value] if isinstance(value, str) else value
        elif key == "precision":
            value = C.PRECISIONS[value] if isinstance(value, str) else value
        elif key == "velocity_integration" and isinstance(value, str):
            value = {"same": -1, "numerical": 0, "analytical": 1}[value]
        if not hasattr(self._c, key):
            raise KeyError(key)
        setattr(self._c, key, value)

    def __getitem__(self, key):
        return getattr(self._c, key)

    def __getattr__(self, key):
        if key.startswith("_"):
            raise AttributeError(key)
        return getattr(self._c, key)

    @classmethod
    def from_ini(cls, params, **kw):
        """From formats.read_config() output (reference key names)."""
        c = cls(
            number_of_timesteps=params["NUMBER_OF_TIMESTEPS"],
            state_save_interval=params["STATE_SAVE_INTERVAL"],
            velocity_save_interval=params["VELOCITY_SAVE_INTERVAL"],
            timestep=params["TIMESTEP"],
            slenderness=params["SLENDERNESS"],
            number_of_terms_in_force_expansion=params["NUMBER_OF_TERMS_IN_FORCE_EXPANSION"],
            number_of_quadrature_intervals=params["NUMBER_OF_QUADRATURE_INTERVALS"],
            number_of_quadrature_points_per_interval=params["NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL"],
            gmres_restart=params["GMRES_RESTART"],
            gmres_max_iterations=params["GMRES_MAX_ITERATIONS"],
            gmres_tolerance=params["GMRES_TOLERANCE"],
            bicgstab_max_iterations=params["BICGSTAB_MAX_ITERATIONS"],
            bicgstab_tolerance=params["BICGSTAB_TOLERANCE"],
        )
        for k, v in kw.items():
            c[k] = v
        return c


class Simulation:
    def __init__(self, config, positions, orientations, allow_noconv=False):
        self._lib = C.load()
        pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        ori = np.ascontiguousarray(orientations, np.float64).reshape(-1, 3)
        if pos.shape != ori.shape:
            raise ValueError("positions and orientations differ in shape")
        self.N = pos.shape[0]
        self.config = config if isinstance(config, Config) else Config(**config)
        M = self.config.number_of_terms_in_force_expansion
        self.R = 3 * M * self.N
        self.allow_noconv = allow_noconv
        h = ctypes.c_void_p()
        C.check(self._lib.rf_create(ctypes.byref(self.config._c), self.N, C.ptr(pos), C.ptr(ori), ctypes.byref(h)),
                "rf_create")
        self._h = h

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.rf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the reference's step seam (src/simulation.h:86-89) ------------------
    def assembleSystem(self):
        C.check(self._lib.rf_assemble(self._h), "assembleSystem")

    def solveSystem(self):
        allow = (C.RF_E_NOCONV,) if self.allow_noconv else ()
        return C.check(self._lib.rf_solve(self._h), "solveSystem", allow)

    def updateVelocities(self):
        C.check(self._lib.rf_update_velocities(self._h), "updateVelocities")

    def updateFibers(self, first_timestep):
        C.check(self._lib.rf_update_fibers(self._h, int(bool(first_timestep))), "updateFibers")

    def step(self, current_timestep):
        allow = (C.RF_E_NOCONV,) if self.allow_noconv else ()
        return C.check(self._lib.rf_step(self._h, int(current_timestep)), "step", allow)

    def run(self, nsteps, first_timestep=0):
        for t in range(first_timestep, first_timestep + nsteps):
            self.step(t)

    # snake_case aliases
    assemble_system = assembleSystem
    solve_system = solveSystem
    update_velocities = updateVelocities
    update_fibers = updateFibers

    # -- state and dumps ----------------------------------------------------
    def state(self):
        pos = np.zeros(3 * self.N)
        ori = np.zeros(3 * self.N)
        C.check(self._lib.rf_get_state(self._h, C.ptr(pos), C.ptr(ori)), "rf_get_state")
        return pos.reshape(-1, 3), ori.reshape(-1, 3)

    def set_state(self, positions, orientations):
        pos = C.f64(positions, 3 * self.N)
        ori = C.f64(orientations, 3 * self.N)
        C.check(self._lib.rf_set_state(self._h, C.ptr(pos), C.ptr(ori)), "rf_set_state")

    def velocities(self):
        t = np.zeros(3 * self.N)
        r = np.zeros(3 * self.N)
        C.check(self._lib.rf_get_velocities(self._h, C.ptr(t), C.ptr(r)), "rf_get_velocities")
        return t.reshape(-1, 3), r.reshape(-1, 3)

    def system(self, with_matrix=True):
        """(A, b): A column-major (R, R) float32 Fortran-ordered, or None."""
        b = np.zeros(self.R)
        A = np.zeros((self.R, self.R), np.float32, order="F") if with_matrix else None
        C.check(self._lib.rf_get_system(self._h, C.ptr(A) if A is not None else None, C.ptr(b)), "rf_get_system")
        return A, b

    def solution(self):
        x = np.zeros(self.R)
        C.check(self._lib.rf_get_solution(self._h, C.ptr(x)), "rf_get_solution")
        return x

    def apply_operator(self, x, which=0):
        """y = A x with the assembled operator (which=1: the 16-bit copy)."""
        xx = C.f64(x, self.R)
        y = np.zeros(self.R)
        C.check(self._lib.rf_operator_apply(self._h, C.ptr(xx), C.ptr(y), int(which)), "rf_operator_apply")
        return y

    def prepare_step_graphs(self, which=3):
        """Build the whole-step graphs now (1 first step, 2 second-order steps,
        3 both; rf_prepare_step_graphs) instead of on a step's second use."""
        C.check(self._lib.rf_prepare_step_graphs(self._h, int(which)), "rf_prepare_step_graphs")

    def set_near_field_preconditioner(self, neighbours):
        """Right-precondition the solve with each fiber's rows of the inverse
        of its neighbourhood block (k nearest fibers, 1..8; 0 off;
        rf_set_near_field_preconditioner); takes effect at the next assembly."""
        C.check(self._lib.rf_set_near_field_preconditioner(self._h, int(neighbours)),
                "rf_set_near_field_preconditioner")

    def set_cuda_graphs(self, mode):
        """0: no CUDA graphs; 1: each rf_step one graph (default); 2: graphs for
        the GMRES restart cycles only, so that the stage times are measured."""
        C.check(self._lib.rf_set_cuda_graphs(self._h, int(mode)), "rf_set_cuda_graphs")

    def autotune(self):
        """Time the matvec and assembly launch choices on the assembled operator
        and keep the fastest (rf_autotune); assembles first if needed."""
        t = C.rf_tune_report()
        rc = self._lib.rf_autotune(self._h, ctypes.byref(t))
        if rc == C.RF_E_STATE:
            self.assembleSystem()
            rc = self._lib.rf_autotune(self._h, ctypes.byref(t))
        C.check(rc, "rf_autotune")
        return {"matvec_variant": t.matvec_variant, "matvec_ms": list(t.matvec_ms),
                "gemv_ctas_per_sm": t.gemv_ctas_per_sm, "gemv_ms": list(t.gemv_ms), "cached": bool(t.cached),
                "panel_blocks": t.panel_blocks, "panel_ms": list(t.panel_ms),
                "asm_variant": t.asm_variant, "asm_ms": list(t.asm_ms)}

    # -- checkpoint / resume ---------------------------------------------------
    def checkpoint(self):
        """The run's resumable state as bytes (rf_checkpoint_save)."""
        n = self._lib.rf_checkpoint_bytes(self._h)
        buf = np.empty(n, np.uint8)
        C.check(self._lib.rf_checkpoint_save(self._h, C.ptr(buf), n), "rf_checkpoint_save")
        return buf.tobytes()

    def restore(self, data):
        """Load a checkpoint taken with the same configuration and fiber count;
        returns the number of steps it had taken (the next step's index)."""
        buf = np.frombuffer(data, np.uint8)
        steps = ctypes.c_int64()
        C.check(self._lib.rf_checkpoint_load(self._h, C.ptr(buf), buf.size, ctypes.byref(steps)),
                "rf_checkpoint_load")
        return steps.value

    def save_checkpoint(self, path):
        with open(path, "wb") as fh:
            fh.write(self.checkpoint())

    def load_checkpoint(self, path):
        with open(path, "rb") as fh:
            return self.restore(fh.read())

    def stats(self):
        s = C.rf_stats()
        C.check(self._lib.rf_last_stats(self._h, ctypes.byref(s)), "rf_last_stats")
        return {k: getattr(s, k) for k, _ in C.rf_stats._fields_}


# -- packed solves of many small suspensions --------------------------------
def _handles(sims):
    arr = (ctypes.c_void_p * len(sims))()
    for k, s in enumerate(sims):
        arr[k] = s._h
    return arr


def solve_packed(sims, allow_noconv=False):
    """Solve the assembled systems of several small mixed-precision
    suspensions with one launch (rf_solve_packed)."""
    lib = C.load()
    allow = (C.RF_E_NOCONV,) if allow_noconv else ()
    return C.check(lib.rf_solve_packed(_handles(sims), len(sims)), "rf_solve_packed", allow)


def step_packed(sims, timesteps):
    """One time step of several small suspensions with a packed solve
    (rf_step_packed); returns the per-suspension status codes."""
    lib = C.load()
    ts = (ctypes.c_int * len(sims))(*[int(t) for t in timesteps])
    st = (ctypes.c_int * len(sims))()
    rc = lib.rf_step_packed(_handles(sims), ts, len(sims), st)
    codes = list(st)
    if rc not in (C.RF_OK, C.RF_E_NOCONV) and all(c == C.RF_OK for c in codes):
        C.check(rc, "rf_step_packed")
    return codes
