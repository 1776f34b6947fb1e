"""Benchmark of the rigid-fiber time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--fibers 4000] [--radius 18] [--precision auto|fp32|mixed_fp16|mixed_bf16]

A "step" is the reference's time step (src/simulation.cu:286-329):
assemble -> solve -> update velocities -> update fibers, on a seeded
synthetic sphere layout (N fibers, centres uniform in a ball of radius R,
min centre distance 0.2, orientations uniform on S^2; M=5, 8x3 quadrature,
eps=0.01, dt=0.1, numerical integration, GMRES tol 1e-5).  Multi-GPU runs are
independent replicas (one per rank, no collective on the data path); value
is the whole-job fiber-steps/s over the max time across ranks.

Prints ONE JSON line on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "fiber-steps/s @N=4000 mixed vs FP32 (err<=1e-4 vs FP64); served p50/p99 step lat"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fibers", type=int, default=4000)
    ap.add_argument("--radius", type=float, default=18.0)
    ap.add_argument("--precision", default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--mixed-restart", type=int, default=20,
                    help="Arnoldi steps between FP64 residual corrections in mixed precision (0: GMRES restart)")
    ap.add_argument("--serve-requests", type=int, default=512,
                    help="suspensions in the served ensemble (0: skip the serving leg)")
    ap.add_argument("--serve-max-active", type=int, default=16)
    ap.add_argument("--serve-rate", type=float, default=400.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-graphs", type=int, default=1, help="replay GMRES cycles from CUDA graphs (1) or not (0)")
    ap.add_argument("--serve-pack-fibers", type=int, default=0,
                    help="requests of at most this many fibers step together with packed solves (0: off)")
    ap.add_argument("--serve-pack-compare", type=int, default=64,
                    help="also run the ensemble with packed solves for requests of at most this many fibers, "
                         "reported as serving_packed (0: skip)")
    ap.add_argument("--direct-fibers", type=int, default=2000,
                    help="fibers of the direct-solver leg (0: skip it)")
    ap.add_argument("--legs", default="headline,serving,direct",
                    help="comma-separated subset of headline,serving,direct; a subset other than the default "
                         "prints the requested legs only (for profiling one part)")
    return ap.parse_args()


def workload(args):
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    pos, ori = sphere_layout(args.fibers, args.radius, 0.2, seed=layout_seed(3, args.fibers))
    return pos, ori


def workload_name(args):
    return ("N=%d fibers in a sphere of radius %g (min centre distance 0.2, S^2 orientations), M=5, 8x3 "
            "quadrature, eps=0.01, dt=0.1, numerical integration, GMRES(10) tol 1e-5" % (args.fibers, args.radius))


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun env); replicas, no collective on the data
    path: only the barrier around the timed region and the max / sum of the
    per-rank results.  NCCL on GPUs, gloo on the host (tests)."""

    def __init__(self, want, backend=None):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.dev = "cuda"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.dev = "cuda" if backend == "nccl" else "cpu"
            if self.dev == "cuda":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def _reduce(self, v, op):
        import torch
        t = torch.tensor([float(v)], device=self.dev, dtype=torch.float64)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self):
        if self.pg:
            import torch
            self._reduce(0.0, self.pg.ReduceOp.SUM)
            if self.dev == "cuda":
                torch.cuda.synchronize()

    def max(self, v):
        return self._reduce(v, self.pg.ReduceOp.MAX) if self.pg else v

    def sum(self, v):
        return self._reduce(v, self.pg.ReduceOp.SUM) if self.pg else v

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def whole_job_rate(dist, local_ms, local_units):
    """(slowest rank's ms, units of all ranks, units per second of the whole job)."""
    ms_max = dist.max(local_ms)
    total = dist.sum(local_units)
    return ms_max, total, total / (ms_max / 1000.0)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# Nominal per-GPU peaks for the kernels that the measured peaks (HBM copy,
# BF16 GEMM) do not cover: FP32 SIMT = 148 SMs x 128 FMA/clock x 2 x 1965 MHz,
# dense TF32 tensor throughput as NVIDIA states it for B200.
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
NOMINAL_TF32_TFLOPS = 1100.0


def asm_flops_per_ordered_pair(M=5, Q=24):
    """The reference algorithm's assembly work per ordered fiber pair (K at
    every (q_i, q_j), 6M + 9 multiply-adds into G and GF, the k_i x k_j
    projections and the block formation); this build evaluates K once per
    unordered pair and folds mirror points, so it executes fewer."""
    return Q * Q * (25 + 2 * 6 * M + 18) + 2 * M * M * Q * 6 + 2 * M * Q * 3 + 25 * 27


def kernel_rooflines(N, head, hbm, mixed, direct=None):
    """Per-stage figures of the timed step (stage times from the timed pass):
    the assembly as reference-algorithm FLOP/s against nominal FP32 and as
    store bandwidth, the velocities from the stored blocks as read bandwidth,
    the LU as 2/3 R^3 against nominal TF32, and the step as the sum of its
    stages' bound times over the measured time."""
    steps = max(head["steps"], 1)
    st = {k: v / steps for k, v in head["stage"].items()}
    pairs = N * (N - 1) / 2.0
    asm_flops = asm_flops_per_ordered_pair() * N * (N - 1)
    t_asm = st["assemble_system"] / 1e3
    out = {"assembly": {"flops_per_ordered_pair": asm_flops_per_ordered_pair(),
                        "achieved_tflops_equivalent": asm_flops / t_asm / 1e12 if t_asm else None,
                        "peak_tflops": NOMINAL_FP32_TFLOPS, "peak_kind": "nominal FP32 SIMT",
                        "frac": asm_flops / t_asm / 1e12 / NOMINAL_FP32_TFLOPS if t_asm else None,
                        "note": "above 1: K is evaluated once per unordered pair and mirror quadrature points "
                                "are folded, so fewer flops run than the reference algorithm counts"}}
    iters = head["iters"] / steps
    if mixed:
        store = pairs * (216 * 4 + 152 * 2)      # FP32 blocks + 16-bit records per unordered pair
        vel_bytes = pairs * 20 * 6 * 4           # rows and columns P0, P1 of the FP32 blocks
        mv_bytes = pairs * 150 * 2
        res_bytes = pairs * 150 * 4
        refs = head["refinements"] / steps
    else:
        store = 4.0 * (15 * N) ** 2
        vel_bytes = None
        mv_bytes = 4.0 * (15 * N) ** 2
        res_bytes = 0.0
        refs = 0.0
    out["assembly"]["store_gbs"] = store / t_asm / 1e9 if t_asm else None
    t_vel = st["update_velocities"] / 1e3
    if vel_bytes:
        out["velocities"] = {"bytes": vel_bytes, "achieved_gbs": vel_bytes / t_vel / 1e9 if t_vel else None,
                             "peak_gbs": hbm, "frac": vel_bytes / t_vel / 1e9 / hbm if t_vel else None}
    bound_ms = 1e3 * (asm_flops / (NOMINAL_FP32_TFLOPS * 1e12) + (iters * mv_bytes + refs * res_bytes) / (hbm * 1e9) +
                      (vel_bytes or 0.0) / (hbm * 1e9))
    step_ms = head["ms"] / steps
    out["step"] = {"bound_ms": bound_ms, "measured_ms": step_ms, "frac": bound_ms / step_ms if step_ms else None,
                   "bound": "assembly at nominal FP32 (reference flops) + matvecs and residuals at measured HBM"}
    if direct and "direct" in direct:
        tf = direct["direct"].get("tflops")
        out["lu"] = {"fibers": direct["fibers"], "achieved_tflops": tf, "peak_tflops": NOMINAL_TF32_TFLOPS,
                     "peak_kind": "nominal dense TF32", "frac": tf / NOMINAL_TF32_TFLOPS if tf else None}
    return out


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a C++ restatement of the reference's Fortran
# path; the Fortran itself cannot be built here) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_sample(pos, ori, iterations, cycles, target_s):
    from oracle import oracle as O
    p = O.Params()
    N = pos.shape[0]
    R = 15 * N
    threads = O.lib().rfo_num_threads()
    rng = np.random.default_rng(0)
    coeff = (1e-3 * rng.standard_normal(R)).astype(np.float32)

    def rows_cost(ns):
        t0 = time.perf_counter()
        slab, _ = O.assemble_rows(pos, ori, p, 0, ns, dtype=np.float32)
        t1 = time.perf_counter()
        O.update_velocities(pos, ori, coeff, p, 0, ns, dtype=np.float32)
        t2 = time.perf_counter()
        xg = rng.standard_normal(R).astype(np.float32)
        reps = 3
        t3 = time.perf_counter()
        for _ in range(reps):
            O.gemv(slab, xg)
        t4 = time.perf_counter()
        return t1 - t0, t2 - t1, (t4 - t3) / reps

    ns = max(1, min(N, threads))
    ta, tv, tg = rows_cost(ns)
    per = (ta + tv + (iterations + cycles) * tg) / ns
    ns2 = int(min(N, max(ns, target_s / max(per, 1e-9))))
    if ns2 > ns:
        ns = ns2
        ta, tv, tg = rows_cost(ns)
    scale = N / ns
    step_s = scale * (ta + tv + (iterations + cycles) * tg)
    t0 = time.perf_counter()
    z = np.zeros((N, 3), np.float32)
    O.update_fibers(False, 0.1, pos.astype(np.float32), pos.astype(np.float32), ori.astype(np.float32),
                    ori.astype(np.float32), z, z, z, z)
    step_s += time.perf_counter() - t0
    return {
        "value": N / step_s, "unit": "fiber-steps/s", "cores": threads, "kind": "port",
        "sample": ("C++ restatement of the reference's Fortran/OpenMP step (FP32, OpenMP over fibers): assembly and "
                   "velocity rows of %d of %d fibers and a dense FP32 gemv over that row slab, scaled by N/%d; "
                   "%d GMRES matvecs per step (iterations + restart residuals, from the GPU run)"
                   % (ns, N, ns, iterations + cycles)),
        "seconds_per_step": step_s,
        "breakdown_s": {"assemble_system": scale * ta, "update_velocities": scale * tv,
                        "solve_system": scale * (iterations + cycles) * tg},
    }


def run_reference(args):
    pos, ori = workload(args)
    iters = 20
    cycles = 3
    for _ in range(args.warmup):
        cpu_sample(pos, ori, iters, cycles, 2.0)
    vals = []
    for _ in range(args.steps):
        vals.append(cpu_sample(pos, ori, iters, cycles, max(1.0, args.cpu_seconds / 2)))
    v = statistics.median(r["value"] for r in vals)
    last = vals[-1]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "fiber-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.fibers / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args), "fibers": args.fibers, "radius": args.radius,
                   "assumed_gmres_matvecs_per_step": iters + cycles},
        "cpu_baseline": {k: last[k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "fiber-steps/s"},
        "e2e": {"value": v, "unit": "fiber-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def time_path(args, dist, cfg, pos, ori, clocks=None):
    """Warm-up, K profiled steps (CUDA events around every matvec launch: the
    roofline figures), then the same K steps again from a checkpoint taken
    after the warm-up, device-timed with the library's defaults (no per-launch
    events, GMRES cycles replayed as CUDA graphs; CUDA events on the handle's
    stream)."""
    import ctypes

    import torch

    from rigidfibers_b200 import Simulation
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    sim = Simulation(cfg, pos, ori)
    sp = ctypes.c_void_p()
    lib.rf_get_stream(sim._h, ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    for t in range(args.warmup):
        sim.step(t)
    tuned = sim.autotune()          # matvec launch choice, timed on this operator
    after_warmup = sim.checkpoint()
    acc = {"stage": {"assemble_system": 0.0, "solve_system": 0.0, "update_velocities": 0.0, "update_fibers": 0.0},
           "iters": 0, "restarts": 0, "refinements": 0, "launches": 0, "mv_launches": 0, "mv_ms": 0.0, "relres": 0.0,
           "graph_replays": 0}
    t = args.warmup
    lib.rf_set_profiling(sim._h, 1)
    for _ in range(args.steps):
        sim.step(t)
        t += 1
        nl, tm = ctypes.c_int(), ctypes.c_double()
        lib.rf_matvec_profile(sim._h, ctypes.byref(nl), ctypes.byref(tm))
        acc["mv_launches"] += nl.value
        acc["mv_ms"] += tm.value
    lib.rf_set_profiling(sim._h, 0)
    t = sim.restore(after_warmup)
    dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sim.step(t)
        t += 1
        st = sim.stats()
        for k in acc["stage"]:
            acc["stage"][k] += st["ms_" + k]
        acc["iters"] += st["iterations"]
        acc["restarts"] += st["restarts"]
        acc["refinements"] += st["refinement_steps"]
        acc["launches"] += st["kernel_launches"]
        acc["graph_replays"] += st["graph_replays"]
        acc["relres"] = max(acc["relres"], st["relative_residual"])
    e1.record(stream)
    torch.cuda.synchronize()
    acc["clocks"] = clocks.stop() if clocks else None
    dist.barrier()
    acc["ms"] = e0.elapsed_time(e1)
    acc["device_bytes"] = sim.stats()["device_bytes"]
    acc["autotune"] = tuned
    sim.close()
    return acc


def e2e_path(args, dist, cfg, pos, ori):
    """Through the C ABI with host buffers: every step uploads the fiber state
    from pinned host memory and reads the new state back (W untimed rounds of
    the same loop first, so the timed steps replay captured graphs as the
    device-timed ones do).  Returns (max seconds over ranks, GMRES iterations
    per step)."""
    import ctypes

    import torch

    from rigidfibers_b200 import Simulation
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    hpos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).pin_memory()
    hori = torch.from_numpy(np.ascontiguousarray(ori, np.float64)).pin_memory()
    out_pos = torch.empty_like(hpos).pin_memory()
    out_ori = torch.empty_like(hori).pin_memory()
    sim = Simulation(cfg, pos, ori)
    sim.step(0)

    def one(t):
        C.check(lib.rf_set_state(sim._h, ctypes.c_void_p(hpos.data_ptr()), ctypes.c_void_p(hori.data_ptr())),
                "rf_set_state")
        sim.step(t)
        C.check(lib.rf_get_state(sim._h, ctypes.c_void_p(out_pos.data_ptr()), ctypes.c_void_p(out_ori.data_ptr())),
                "rf_get_state")
        return sim.stats()["iterations"]

    for t in range(1, 1 + args.warmup):
        one(t)
    dist.barrier()
    torch.cuda.synchronize()
    iters = 0
    t0 = time.perf_counter()
    for t in range(1 + args.warmup, 1 + args.warmup + args.steps):
        iters += one(t)
    torch.cuda.synchronize()
    s = dist.max(time.perf_counter() - t0)
    sim.close()
    return s, iters / args.steps


def error_vs_fp64(precision, n=300):
    """Relative error of the given path against the FP64 oracle (direct
    solve) on a seeded layout of n fibers at the workload's density, 2 steps."""
    from oracle import oracle as O
    from rigidfibers_b200 import Config, Simulation
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    radius = 18.0 * (n / 4000.0) ** (1.0 / 3.0)
    pos, ori = sphere_layout(n, radius, 0.2, seed=layout_seed(3, n))
    ref = O.run_steps(pos, ori, O.Params(), 2, solver="direct", dtype=np.float64)
    sim = Simulation(Config(precision=precision), pos, ori)
    err = {"fibers": n, "steps": 2}
    for t in range(2):
        sim.assembleSystem()
        sim.solveSystem()
        x = sim.solution()
        sim.updateVelocities()
        tv, rv = sim.velocities()
        sim.updateFibers(t == 0)
        p1, o1 = sim.state()
        for k, v in (("forces", x), ("tvel", tv), ("rvel", rv), ("pos", p1), ("ori", o1)):
            r = np.asarray(ref[t][{"forces": "x"}.get(k, k)]).reshape(-1)
            e = float(np.abs(np.asarray(v).reshape(-1) - r).max() / np.abs(r).max())
            err[k] = max(err.get(k, 0.0), e)
    sim.close()
    return err


def serve_ensemble(args, dist, pack_fibers=None):
    """The served ensemble: independent suspensions (N log-uniform in
    [16, 1000], eps in {0.01, 0.005}, 5-50 steps, BF16 pair blocks) arriving
    as a Poisson stream into one rf_server; per-step latency percentiles and
    aggregate fiber-steps/s over the whole run (first submit -> last result)."""
    from rigidfibers_b200 import Config
    from rigidfibers_b200.generate import request_layout, serving_requests
    from rigidfibers_b200.server import Server

    reqs = serving_requests(args.serve_requests, seed=11 + dist.rank)
    layouts = [request_layout(r) for r in reqs]
    cfgs = [Config(slenderness=r["slenderness"], precision="mixed_bf16", refinement_restart=args.mixed_restart)
            for r in reqs]
    rng = np.random.default_rng(5 + dist.rank)
    gaps = rng.exponential(1.0 / args.serve_rate, size=len(reqs))
    dist.barrier()
    pack = args.serve_pack_fibers if pack_fibers is None else pack_fibers
    with Server(max_active=args.serve_max_active, use_cuda_graphs=args.serve_graphs, pack_max_fibers=pack) as srv:
        t0 = time.perf_counter()
        due = t0
        for r, (p, o), c, g in zip(reqs, layouts, cfgs, gaps):
            due += g
            delay = due - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            srv.submit(c, p, o, r["nsteps"])
        srv.drain()
        wall = time.perf_counter() - t0
        st = srv.stats()
    dist.barrier()
    wall_max = dist.max(wall)
    fiber_steps = dist.sum(st["fiber_steps"])
    return {"requests": len(reqs) * dist.world, "completed": int(dist.sum(st["completed"])),
            "failed": int(dist.sum(st["failed"])), "steps": int(dist.sum(st["steps"])),
            "p50_step_ms": st["p50_step_ms"], "p99_step_ms": st["p99_step_ms"],
            "fiber_steps_per_s": fiber_steps / wall_max, "wall_s": wall_max, "arrival_rate_per_s": args.serve_rate,
            "max_active": args.serve_max_active, "peak_active": st["peak_active"],
            "cuda_graphs": bool(args.serve_graphs), "pack_max_fibers": pack,
            "peak_device_bytes": st["peak_bytes"], "storage": "mixed_bf16",
            "workload": "N log-uniform in [16, 1000], eps in {0.01, 0.005}, 5-50 steps, volume fraction 1%, "
                        "M=5, 8x3 quadrature, Poisson arrivals; latency = host wall time of one rf_step "
                        "while the others run (rank 0's percentiles)"}


def direct_leg(args):
    """The thesis-scale configuration: N fibers (radius 14 sphere at N=2000),
    analytical integration, one step solved by the blocked LU (in place of
    MAGMA's sgesv) and by GMRES on the same system.  LU rate = 2/3 R^3 flops over
    the solve time (factorisation, triangular solves and FP64 refinement)."""
    from rigidfibers_b200 import Config, Simulation
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    n = args.direct_fibers
    radius = 14.0 * (n / 2000.0) ** (1.0 / 3.0)
    pos, ori = sphere_layout(n, radius, 0.2, seed=layout_seed(2, n))
    out = {"fibers": n, "radius": radius, "integration": "analytical"}
    for solver in ("direct", "gmres"):
        sim = Simulation(Config(solver=solver, integration="analytical"), pos, ori)
        sim.step(0)                      # warm-up (first-touch of the kernels)
        tuned = sim.autotune()
        sim.assembleSystem()
        sim.solveSystem()
        st = sim.stats()
        sim.close()
        R = 15 * n
        leg = {"ms_solve": st["ms_solve_system"], "ms_assemble": st["ms_assemble_system"],
               "relative_residual": st["relative_residual"], "iterations": st["iterations"],
               "refinements": st["refinement_steps"], "autotune": tuned}
        if solver == "direct":
            leg["tflops"] = (2.0 / 3.0) * R ** 3 / (st["ms_solve_system"] / 1e3) / 1e12
        out[solver] = leg
    return out


def run_ours(args, dist):
    import torch

    from rigidfibers_b200 import Config

    torch.cuda.set_device(dist.local)
    pos, ori = workload(args)
    N = args.fibers
    R = 15 * N
    precision = "mixed_fp16" if args.precision == "auto" else args.precision
    cfg = Config(precision=precision, refinement_restart=args.mixed_restart)
    head = time_path(args, dist, cfg, pos, ori, clocks=Clocks(dist.local))
    ms_max, total_fiber_steps, value = whole_job_rate(dist, head["ms"], N * args.steps)
    e2e_s, e2e_iters = e2e_path(args, dist, cfg, pos, ori)
    e2e_value = total_fiber_steps / e2e_s
    # bytes the C ABI moves per step: rf_set_state uploads double4 prev+cur
    # position/orientation and their float4 copies; rf_get_state reads double4 pos/ori
    h2d = N * (2 * 2 * 32 + 2 * 16)
    d2h = N * 2 * 32

    comparison = None
    if precision != "fp32":
        plain = time_path(args, dist, Config(precision="fp32"), pos, ori)
        plain_ms = dist.max(plain["ms"])
        comparison = {"precision": "fp32", "value": total_fiber_steps / (plain_ms / 1000.0),
                      "ms_per_step": plain_ms / args.steps,
                      "stage_ms_per_step": {k: v / args.steps for k, v in plain["stage"].items()},
                      "gmres_iterations_per_step": plain["iters"] / args.steps,
                      "matvec_ms": plain["mv_ms"] / max(plain["mv_launches"], 1),
                      "autotune": plain["autotune"]}

    hbm, peak_kind = peaks()
    mvn = max(head["mv_launches"], 1)
    mv_avg_ms = head["mv_ms"] / mvn
    if precision == "fp32":
        kernel = "k_gemv_cm_f32 (dense FP32 column-major matvec, GMRES)"
        bytes_per_matvec = 4.0 * R * R
    else:
        kernel = ("k_struct_z16_bulk<5> + k_sum_parts + k_struct_finalize (16-bit structured matvec, "
                  "TMA bulk-copy pipeline, GMRES)")
        bytes_per_matvec = 2.0 * 150 * N * (N - 1) / 2
    achieved = bytes_per_matvec / (mv_avg_ms / 1000.0) / 1e9 if head["mv_launches"] else None
    # DRAM traffic per launch from one ncu capture of the same kernel at N=1500
    # (dram__bytes_read.sum 347.6 MB + dram__bytes_write.sum 9.8 MB for 1124250
    # unordered pairs: 304-byte records for 300 algorithmic bytes, x, partial
    # rows; profiles/struct_z16_bulk_N1500.md), scaled by the pairs one launch
    # processes; not captured for the dense FP32 kernel
    traffic = 357.4e6 / (1500 * 1499 / 2) * (N * (N - 1) / 2) if precision != "fp32" else None
    roof = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": hbm, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
            "traffic_source": "ncu capture at N=1500 scaled by pairs" if traffic else None,
            "algorithmic_bytes_per_launch": bytes_per_matvec, "avg_launch_ms": mv_avg_ms,
            "launches": head["mv_launches"], "share_of_step_time": head["mv_ms"] / head["ms"] if head["ms"] else None,
            "measured_in": "a profiled pass of the same K steps just before the timed ones (CUDA events around "
                           "each matvec launch on the handle's stream; per-launch events rule out graph replay)"}
    out = {
        "metric": METRIC, "value": value, "unit": "fiber-steps/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if precision == "fp32" else "%s storage, f32 accumulate, f64 refinement" % precision[6:],
        "data": "synthetic",
        "config": {"workload": workload_name(args), "fibers": N, "radius": args.radius, "precision": precision,
                   "parallelism": "replicas x%d" % dist.world,
                   "l2": "inputs larger than L2: the operator (%.1f GB) is re-assembled and re-read every step"
                         % (head["device_bytes"] / 1e9)},
        "stage_ms_per_step": {k: v / args.steps for k, v in head["stage"].items()},
        "gmres_iterations_per_step": head["iters"] / args.steps,
        "gmres_restarts_per_step": head["restarts"] / args.steps,
        "refinements_per_step": head["refinements"] / args.steps,
        "graph_replays_per_step": head["graph_replays"] / args.steps,
        "max_relative_residual": head["relres"],
        "roofline": roof, "clocks": head["clocks"],
        "e2e": {"value": e2e_value, "unit": "fiber-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "gmres_iterations_per_step": e2e_iters,
                "timing": "host wall clock, max over ranks; every step uploads the initial layout from pinned host "
                          "memory (rf_set_state) and reads the new state back (rf_get_state)"},
        "gpu_launches": head["launches"],
        "autotune": head["autotune"],
    }
    if args.serve_requests > 0:
        out["serving"] = serve_ensemble(args, dist)
        if args.serve_pack_compare > 0 and args.serve_pack_compare != args.serve_pack_fibers:
            out["serving_packed"] = serve_ensemble(args, dist, args.serve_pack_compare)
    if args.direct_fibers > 0 and dist.rank == 0:
        out["direct_solver"] = direct_leg(args)
    if comparison:
        out["fp32_path"] = comparison
        out["speedup_vs_fp32"] = value / comparison["value"]
    head["steps"] = args.steps
    out["kernels"] = kernel_rooflines(N, head, hbm, precision != "fp32", out.get("direct_solver"))
    if dist.rank == 0 and not args.no_cpu_baseline:
        out["error_vs_fp64"] = error_vs_fp64(precision)
        # the CPU port runs the reference's FP32 GMRES: its matvec count is the FP32 path's
        src = plain if comparison else head
        out["cpu_baseline"] = cpu_sample(pos, ori, max(1, src["iters"] // args.steps),
                                         max(1, src["restarts"] // args.steps), args.cpu_seconds)
    if dist.rank == 0:
        print(json.dumps(out), flush=True)


def run_legs(args, dist):
    """Only the legs named in --legs (no headline metric line)."""
    import torch
    torch.cuda.set_device(dist.local)
    legs = set(args.legs.split(","))
    out = {"legs": sorted(legs)}
    if "serving" in legs:
        out["serving"] = serve_ensemble(args, dist)
        if args.serve_pack_compare > 0 and args.serve_pack_compare != args.serve_pack_fibers:
            out["serving_packed"] = serve_ensemble(args, dist, args.serve_pack_compare)
    if "direct" in legs and dist.rank == 0:
        out["direct_solver"] = direct_leg(args)
    if dist.rank == 0:
        print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        # the reference arm runs on host cores only; ranks > 0 exit without work
        if int(os.environ.get("RANK", "0")) == 0:
            run_reference(args)
        return
    dist = Dist(args.gpus)
    try:
        if "headline" in args.legs.split(","):
            if "serving" not in args.legs.split(","):
                args.serve_requests = 0
            if "direct" not in args.legs.split(","):
                args.direct_fibers = 0
            run_ours(args, dist)
        else:
            run_legs(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
