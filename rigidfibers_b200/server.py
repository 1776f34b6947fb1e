"""Serving loop for ensembles of independent suspensions over the C ABI
(rf_server_* in include/rigidfibers.h).

    with Server(max_active=16) as srv:
        rid = srv.submit(Config(...), positions, orientations, nsteps=20)
        srv.wait(rid)
        pos, ori, tvel, rvel, st = srv.result(rid)
        print(srv.stats()["p99_step_ms"])

The reference runs one suspension per process (fibers_runner.py:17-162);
here many suspensions share one GPU: admission in arrival order by free slot
and device-memory budget, one handle and stream per running suspension; with
pack_max_fibers > 0 the small ones step together, their systems solved by
a few launches per step (rf_step_packed).
"""
import ctypes

import numpy as np

from . import _capi as C
from .simulation import Config

STATUS = {C.RF_REQ_QUEUED: "queued", C.RF_REQ_RUNNING: "running", C.RF_REQ_DONE: "done",
          C.RF_REQ_FAILED: "failed", C.RF_REQ_CANCELLED: "cancelled"}


def device_bytes(config, number_of_fibers):
    """Device memory a handle of this configuration allocates."""
    lib = C.load()
    cfg = config if isinstance(config, Config) else Config(**config)
    n = lib.rf_device_bytes_estimate(ctypes.byref(cfg._c), int(number_of_fibers))
    if n < 0:
        raise ValueError("invalid configuration for %d fibers" % number_of_fibers)
    return int(n)


class Server:
    def __init__(self, max_active=None, hbm_budget_bytes=None, use_cuda_graphs=None, pack_max_fibers=None,
                 pack_max_members=None, reserve_bytes=None):
        self._lib = C.load()
        sc = C.rf_server_config()
        C.check(self._lib.rf_server_config_default(ctypes.byref(sc)), "rf_server_config_default")
        if max_active is not None:
            sc.max_active = int(max_active)
        if hbm_budget_bytes is not None:
            sc.hbm_budget_bytes = int(hbm_budget_bytes)
        if use_cuda_graphs is not None:
            # True / False as before; an int is the rf_set_cuda_graphs mode (0, 1 or 2)
            sc.use_cuda_graphs = (2 if use_cuda_graphs else 0) if isinstance(use_cuda_graphs, bool) else \
                int(use_cuda_graphs)
        if pack_max_fibers is not None:
            sc.pack_max_fibers = int(pack_max_fibers)
        if pack_max_members is not None:
            sc.pack_max_members = int(pack_max_members)
        if reserve_bytes is not None:
            sc.reserve_bytes = int(reserve_bytes)
        self.pack_max_fibers = sc.pack_max_fibers
        self.max_active = sc.max_active
        self.hbm_budget_bytes = sc.hbm_budget_bytes
        s = ctypes.c_void_p()
        C.check(self._lib.rf_server_create(ctypes.byref(sc), ctypes.byref(s)), "rf_server_create")
        self._s = s
        self._n = {}

    def submit(self, config, positions, orientations, nsteps):
        cfg = config if isinstance(config, Config) else Config(**config)
        pos = np.ascontiguousarray(positions, np.float64).reshape(-1, 3)
        ori = np.ascontiguousarray(orientations, np.float64).reshape(-1, 3)
        if pos.shape != ori.shape:
            raise ValueError("positions and orientations differ in shape")
        rid = ctypes.c_int64()
        C.check(self._lib.rf_server_submit(self._s, ctypes.byref(cfg._c), pos.shape[0], C.ptr(pos), C.ptr(ori),
                                           int(nsteps), ctypes.byref(rid)), "rf_server_submit")
        self._n[rid.value] = pos.shape[0]
        return rid.value

    def poll(self, rid):
        st, done = ctypes.c_int(), ctypes.c_int()
        C.check(self._lib.rf_server_poll(self._s, rid, ctypes.byref(st), ctypes.byref(done)), "rf_server_poll")
        return STATUS[st.value], done.value

    def cancel(self, rid):
        C.check(self._lib.rf_server_cancel(self._s, rid), "rf_server_cancel")

    def wait(self, rid, timeout=600.0):
        C.check(self._lib.rf_server_wait(self._s, rid, float(timeout)), "rf_server_wait")
        return self.poll(rid)[0]

    def drain(self, timeout=3600.0):
        C.check(self._lib.rf_server_drain(self._s, float(timeout)), "rf_server_drain")

    def result(self, rid):
        """(positions, orientations, tvel, rvel, stats) of a finished request."""
        n = self._n[rid]
        out = [np.empty((n, 3), np.float64) for _ in range(4)]
        st = C.rf_request_stats()
        C.check(self._lib.rf_server_result(self._s, rid, *[C.ptr(a) for a in out], ctypes.byref(st)),
                "rf_server_result")
        stats = {k: getattr(st, k) for k, _ in C.rf_request_stats._fields_}
        return out[0], out[1], out[2], out[3], stats

    def step_times(self, rid):
        """Host wall time of each step of a finished request (ms, step order)."""
        n = ctypes.c_int()
        C.check(self._lib.rf_server_step_times(self._s, rid, None, 0, ctypes.byref(n)), "rf_server_step_times")
        out = np.zeros(n.value, np.float64)
        C.check(self._lib.rf_server_step_times(self._s, rid, C.ptr(out), n.value, ctypes.byref(n)),
                "rf_server_step_times")
        return out

    def stats(self):
        st = C.rf_server_stats()
        C.check(self._lib.rf_server_get_stats(self._s, ctypes.byref(st)), "rf_server_get_stats")
        return {k: getattr(st, k) for k, _ in C.rf_server_stats._fields_}

    def close(self):
        if getattr(self, "_s", None):
            self._lib.rf_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
