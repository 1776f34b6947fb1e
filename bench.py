"""Benchmark of the rigid-fiber time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--fibers 4000] [--radius 18] [--precision auto|fp32|mixed_fp16|mixed_bf16|matrix_free|mixed_fp16_recompute]

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
    ap.add_argument("--no-fp32-path", action="store_true",
                    help="skip the plain FP32 comparison legs (the dense matrix of large N does not fit beside)")
    ap.add_argument("--no-error-leg", action="store_true",
                    help="skip the step errors against the FP64 reference at the benchmark configurations")
    ap.add_argument("--reference-cap-s", type=float, default=300.0,
                    help="reference arm: stop timing CPU steps when the next one would end past this many seconds")
    ap.add_argument("--mixed-restart", type=int, default=20,
                    help="Arnoldi steps between FP64 residual corrections in mixed precision (0: GMRES restart)")
    ap.add_argument("--serve-requests", type=int, default=512,
                    help="suspensions in the served ensemble (0: skip the serving leg)")
    ap.add_argument("--serve-max-active", type=int, default=8,
                    help="requests stepping on their own handles at once (the pack's members are not counted)")
    ap.add_argument("--serve-rate", type=float, default=400.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-graphs", type=int, default=2,
                    help="CUDA graph mode of the served requests: 2 restart cycles (default), 1 whole steps built "
                         "at admission, 0 off")
    ap.add_argument("--serve-pack-fibers", type=int, default=128,
                    help="requests of at most this many fibers step together with packed solves (0: off)")
    ap.add_argument("--serve-compare", default="0,16",
                    help="PACK_FIBERS,MAX_ACTIVE: also run the ensemble so (default: no packing, 16 requests at "
                         "once), reported as serving_compare ('': skip)")
    ap.add_argument("--direct-fibers", type=int, default=2000,
                    help="fibers of the direct-solver leg (0: skip it)")
    ap.add_argument("--direct-large-fibers", type=int, default=4000,
                    help="fibers of the direct solve at the precision configuration (numerical; 0: skip it)")
    ap.add_argument("--legs", default="headline,serving,direct",
                    help="comma-separated subset of headline,serving,direct,error,cpu; without headline only the "
                         "requested legs are run and printed (for profiling one part)")
    return ap.parse_args()


def workload_layout(fibers, radius=None):
    """The seeded layout of the precision configuration: N fibers, centres in
    a ball of radius 18 (N=4000; scaled as N^(1/3) by default for other N)."""
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    if radius is None:
        radius = 18.0 * (fibers / 4000.0) ** (1.0 / 3.0)
    return sphere_layout(fibers, radius, 0.2, seed=layout_seed(3, fibers))


def workload(args):
    return workload_layout(args.fibers, args.radius)


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

# Flops the structured assembly kernel k_assemble_pairs<5,24,FP16,numerical>
# executes per unordered fiber pair, from one ncu capture of its scalar variant
# at N=1000 (499,500 pairs): thread instructions FFMA 7.15 G x 2 + FMUL 1.69 G
# + FADD 1.92 G = 17.9 GFLOP.  The kernel evaluates the Stokeslet once per
# unordered pair, folds mirror quadrature points and contracts four scalar
# moments per point, so this is what its FP32 pipes actually do; the
# reference algorithm counts 2 x 67,923 for the same pair.  The packed
# (f32x2) variant executes the same flops in fewer instructions.
ASM_EXEC_FLOPS_PER_PAIR = (7.15e9 * 2 + 1.69e9 + 1.92e9) / 499500.0
# the same capture: 78.5 % of the issue slots busy, FMA pipe 56 %, DRAM 12 %
ASM_BOUND = "FP32 instruction issue (ncu, N=1000: 78.5 % of issue slots busy, FMA pipe 56 %, DRAM 12 %)"


def asm_flops_per_ordered_pair(M=5, Q=24):
    """The reference algorithm's assembly work per ordered fiber pair (K at
    every (q_i, q_j), 6M + 9 multiply-adds into G and GF, the k_i x k_j
    projections and the block formation); this build evaluates K once per
    unordered pair and folds mirror points, so it executes fewer."""
    return Q * Q * (25 + 2 * 6 * M + 18) + 2 * M * M * Q * 6 + 2 * M * Q * 3 + 25 * 27


def kernel_rooflines(N, head, hbm, mixed, direct=None):
    """Per-stage figures of the timed step (stage times from the timed pass):
    the assembly as executed FLOP/s (ncu instruction mix per unordered pair)
    against nominal FP32 SIMT and as store bandwidth, the velocities from the
    stored blocks as read bandwidth, the LU as 2/3 R^3 per second against
    nominal TF32, and the step as the sum of its stages' bound times over the
    measured time."""
    steps = max(head["steps"], 1)
    st = {k: v / steps for k, v in head["stage"].items()}
    pairs = N * (N - 1) / 2.0
    exec_flops = ASM_EXEC_FLOPS_PER_PAIR * pairs
    t_asm = st["assemble_system"] / 1e3
    out = {"assembly": {"executed_flops_per_unordered_pair": ASM_EXEC_FLOPS_PER_PAIR,
                        "achieved_tflops": exec_flops / t_asm / 1e12 if t_asm else None,
                        "peak_tflops": NOMINAL_FP32_TFLOPS, "peak_kind": "nominal FP32 SIMT",
                        "frac": exec_flops / t_asm / 1e12 / NOMINAL_FP32_TFLOPS if t_asm else None,
                        "bound": ASM_BOUND,
                        "reference_flops_per_ordered_pair": asm_flops_per_ordered_pair()}}
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
    bound_ms = 1e3 * (exec_flops / (NOMINAL_FP32_TFLOPS * 1e12) + (iters * mv_bytes + refs * res_bytes) / (hbm * 1e9) +
                      (vel_bytes or 0.0) / (hbm * 1e9))
    step_ms = head["ms"] / steps
    out["step"] = {"bound_ms": bound_ms, "measured_ms": step_ms, "frac": bound_ms / step_ms if step_ms else None,
                   "bound": "assembly's executed flops at nominal FP32 + matvecs and residuals at measured HBM"}
    if direct and "direct" in direct:
        tf = direct["direct"].get("tflops")
        out["lu"] = {"fibers": direct["fibers"], "achieved_tflops": tf, "peak_tflops": NOMINAL_TF32_TFLOPS,
                     "peak_kind": "nominal dense TF32", "frac": tf / NOMINAL_TF32_TFLOPS if tf else None}
    return out


# ---------------------------------------------------------------------------
# CPU: the oracle (a C++ restatement of the reference's Fortran/OpenMP path;
# the Fortran itself cannot be built here), full time steps on the host cores
# ---------------------------------------------------------------------------
def cpu_steps(pos, ori, timed, untimed=1, cap_s=None, analytical=False):
    """The reference's time loop (fortran/fibers.f95:182-349) run by the oracle
    in FP32 on all host cores: per step the full dense assembly (R x R FP32),
    GMRES(10) to 1e-5 with its own iteration count (sgmres semantics), the
    velocities and the fiber update.  `untimed` steps run first (the
    reference's own timers exclude step 0); then up to `timed` timed steps, or
    fewer when the next one would end past cap_s seconds of timed work."""
    from oracle import oracle as O
    p = O.Params()
    f32 = np.float32
    cur_pos = np.array(pos, f32).reshape(-1, 3)
    cur_ori = np.array(ori, f32).reshape(-1, 3)
    prev_pos, prev_ori = cur_pos.copy(), cur_ori.copy()
    prev_tv = np.zeros_like(cur_pos)
    prev_rv = np.zeros_like(cur_pos)
    recs = []
    spent = 0.0
    for t in range(untimed + timed):
        t0 = time.perf_counter()
        A, b = O.assemble(cur_pos, cur_ori, p, analytical, f32)
        t1 = time.perf_counter()
        x, it, rel = O.solve(A, b, p, "gmres")
        t2 = time.perf_counter()
        del A
        tv, rv = O.update_velocities(cur_pos, cur_ori, x, p, dtype=f32, analytical=analytical)
        t3 = time.perf_counter()
        npos, nori = O.update_fibers(t == 0, p.dt, prev_pos, cur_pos, prev_ori, cur_ori, prev_tv, tv, prev_rv, rv)
        t4 = time.perf_counter()
        if t >= untimed:
            recs.append({"assemble_system": t1 - t0, "solve_system": t2 - t1, "update_velocities": t3 - t2,
                         "update_fibers": t4 - t3, "total": t4 - t0, "iterations": it, "relres": rel})
            spent += t4 - t0
            if cap_s is not None and spent + (t4 - t0) > cap_s:
                break
        prev_pos, cur_pos = cur_pos, npos
        prev_ori, cur_ori = cur_ori, nori
        prev_tv, prev_rv = tv, rv
    n = len(recs)
    N = len(cur_pos)
    total = sum(r["total"] for r in recs)
    return {"value": N * n / total, "steps": n, "seconds_per_step": total / n, "cores": O.lib().rfo_num_threads(),
            "stage_s_per_step": {k: sum(r[k] for r in recs) / n
                                 for k in ("assemble_system", "solve_system", "update_velocities", "update_fibers")},
            "gmres_iterations_per_step": sum(r["iterations"] for r in recs) / n,
            "max_relative_residual": max(r["relres"] for r in recs)}


CPU_KIND = "port"
CPU_WHAT = ("the oracle, a C++ restatement of the reference's Fortran/OpenMP time step (FP32, OpenMP over fibers, "
            "full dense assembly, GMRES(10) to 1e-5 with sgmres semantics, velocities, fiber update)")


def one_thread_sample(N, radius, fibers=32):
    """Seconds per step on one host thread, from a bounded sample run in a
    child process with OMP_NUM_THREADS=1: the assembly and velocity rows of
    `fibers` fibers of the N-fiber workload and a GEMV over that row slab,
    scaled by N / fibers (the rest of a step is O(N) or O(R) work)."""
    code = ("import sys, time, json, numpy as np; sys.path.insert(0, %r)\n"
            "from bench import workload_layout\n"
            "from oracle import oracle as O\n"
            "pos, ori = workload_layout(%d, %r)\n"
            "p = O.Params(); ns = %d\n"
            "t0 = time.perf_counter(); slab, _ = O.assemble_rows(pos, ori, p, 0, ns, dtype=np.float32)\n"
            "t1 = time.perf_counter(); O.update_velocities(pos, ori, np.zeros(15 * len(pos), np.float32), p, 0, ns,"
            " dtype=np.float32)\n"
            "t2 = time.perf_counter(); O.gemv(slab, np.ones(slab.shape[1], np.float32)); t3 = time.perf_counter()\n"
            "print(json.dumps({'asm': t1 - t0, 'vel': t2 - t1, 'gemv': t3 - t2, "
            "'threads': O.lib().rfo_num_threads()}))\n") % (ROOT, N, radius, fibers)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    try:
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        d = json.loads(r.stdout.strip().splitlines()[-1])
    except (subprocess.SubprocessError, ValueError, IndexError) as e:
        return {"unavailable": str(e)[:200]}
    return d


def run_reference(args):
    pos, ori = workload(args)
    res = cpu_steps(pos, ori, args.steps, untimed=1, cap_s=args.reference_cap_s)
    v = res["value"]
    one = one_thread_sample(args.fibers, args.radius)
    if "asm" in one:
        scale = args.fibers / 32.0
        s1 = scale * (one["asm"] + one["vel"] + one["gemv"] * (res["gmres_iterations_per_step"] + 3))
        one_thread = {"value": args.fibers / s1, "unit": "fiber-steps/s", "threads": one["threads"],
                      "sample": "assembly and velocity rows of 32 of %d fibers and a GEMV over that slab "
                                "(x %.1f GMRES matvecs per step), scaled by N/32" %
                                (args.fibers, res["gmres_iterations_per_step"] + 3)}
    else:
        one_thread = one
    sample = ("%s; %d full time steps of the N=%d workload timed (step 0, first-order, run untimed first as the "
              "reference's timers exclude it)" % (CPU_WHAT, res["steps"], args.fibers))
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "fiber-steps/s", "n_gpus": args.gpus,
        "steps": res["steps"], "warmup": 1, "ms_per_step": 1000.0 * res["seconds_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args), "fibers": args.fibers, "radius": args.radius,
                   "precision": "fp32", "requested_steps": args.steps, "requested_warmup": args.warmup},
        "cpu_baseline": {"kind": CPU_KIND, "cores": res["cores"], "sample": sample, "value": v,
                         "unit": "fiber-steps/s"},
        "e2e": {"value": v, "unit": "fiber-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "stage_s_per_step": res["stage_s_per_step"],
        "gmres_iterations_per_step": res["gmres_iterations_per_step"],
        "max_relative_residual": res["max_relative_residual"],
        "one_thread": one_thread,
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _stream_of(lib, sim):
    import ctypes

    import torch
    sp = ctypes.c_void_p()
    lib.rf_get_stream(sim._h, ctypes.byref(sp))
    return torch.cuda.ExternalStream(sp.value)


def time_path(args, dist, cfg, pos, ori, clocks=None, profile=True):
    """W warm-up steps and the autotuner, a checkpoint C, two steps that
    capture the step graph (discarded: C is restored), then K steps from C
    device-timed with the library's defaults (each step one CUDA graph, no
    per-launch events; CUDA events on the handle's stream), then the same K
    steps from C again launched stage by stage with CUDA events around every
    matvec launch (the roofline's per-launch figures and the stage times)."""
    import ctypes

    import torch

    from rigidfibers_b200 import Simulation
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    sim = Simulation(cfg, pos, ori)
    stream = _stream_of(lib, sim)
    for t in range(args.warmup):
        sim.step(t)
    tuned = sim.autotune()          # launch choices, timed on this operator
    ckpt = sim.checkpoint()
    t = args.warmup
    for _ in range(3):
        sim.step(t)
        t += 1
    acc = {"stage": {"assemble_system": 0.0, "solve_system": 0.0, "update_velocities": 0.0, "update_fibers": 0.0},
           "iters": 0, "restarts": 0, "refinements": 0, "launches": 0, "mv_launches": 0, "mv_ms": 0.0, "relres": 0.0,
           "graph_replays": 0, "iters_per_step": []}
    t = sim.restore(ckpt)
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
        acc["iters"] += st["iterations"]
        acc["iters_per_step"].append(st["iterations"])
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
    if profile:
        t = sim.restore(ckpt)
        lib.rf_set_profiling(sim._h, 1)
        for _ in range(args.steps):
            sim.step(t)
            t += 1
            # stage times: this pass launches stage by stage (the timed pass
            # runs each step as one graph and reports its total only)
            st = sim.stats()
            for k in acc["stage"]:
                acc["stage"][k] += st["ms_" + k]
            nl, tm = ctypes.c_int(), ctypes.c_double()
            lib.rf_matvec_profile(sim._h, ctypes.byref(nl), ctypes.byref(tm))
            acc["mv_launches"] += nl.value
            acc["mv_ms"] += tm.value
        lib.rf_set_profiling(sim._h, 0)
    acc["device_bytes"] = sim.stats()["device_bytes"]
    acc["autotune"] = tuned
    sim.close()
    return acc


def e2e_path(args, dist, cfg, pos, ori):
    """The same K steps (from the state after the W warm-up steps) through the
    C ABI with the run's state in host memory between steps: every step loads
    the state it needs (positions and orientations of the current and previous
    step, in FP64 and FP32, and the previous velocities: rf_checkpoint_load)
    from pinned host memory, runs rf_step, and reads the next state back
    (rf_checkpoint_save).  Host wall clock, max over ranks.  Returns (seconds,
    GMRES iterations per step, bytes per copy)."""
    import ctypes

    import torch

    from rigidfibers_b200 import Simulation
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    sim = Simulation(cfg, pos, ori)
    for t in range(args.warmup):
        sim.step(t)
    sim.autotune()                  # the cached choice of the device-timed pass
    nbytes = lib.rf_checkpoint_bytes(sim._h)
    host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    start = torch.empty_like(host).pin_memory()
    hp = ctypes.c_void_p(host.data_ptr())
    C.check(lib.rf_checkpoint_save(sim._h, ctypes.c_void_p(start.data_ptr()), nbytes), "rf_checkpoint_save")
    taken = ctypes.c_int64()

    def one():
        C.check(lib.rf_checkpoint_load(sim._h, hp, nbytes, ctypes.byref(taken)), "rf_checkpoint_load")
        sim.step(taken.value)
        C.check(lib.rf_checkpoint_save(sim._h, hp, nbytes), "rf_checkpoint_save")
        return sim.stats()["iterations"]

    host.copy_(start)
    for _ in range(2):              # captures the GMRES graphs; discarded
        one()
    host.copy_(start)
    dist.barrier()
    torch.cuda.synchronize()
    iters = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        iters += one()
    torch.cuda.synchronize()
    s = dist.max(time.perf_counter() - t0)
    sim.close()
    return s, iters / args.steps, int(nbytes)


def fp64_reference_step(pos, ori, analytical=False):
    """One time step (step 0: Euler update) of the reference method in FP64:
    the oracle's FP64 assembly and velocities on the host cores, and the dense
    FP64 system solved on the GPU by LU (torch.linalg.solve) as the checker.
    Returns b, x, tvel, rvel and the next positions / orientations."""
    import torch

    from oracle import oracle as O
    p = O.Params()
    f64 = np.float64
    A, b = O.assemble(pos, ori, p, analytical, f64)
    Ad = torch.from_numpy(A).to("cuda")          # column-major host array -> a transposed-stride tensor
    del A
    x = torch.linalg.solve(Ad, torch.from_numpy(b).to("cuda")).cpu().numpy()
    del Ad
    torch.cuda.empty_cache()
    tv, rv = O.update_velocities(pos, ori, x, p, dtype=f64, analytical=analytical)
    z = np.zeros_like(np.asarray(pos, f64))
    npos, nori = O.update_fibers(True, p.dt, pos, pos, ori, ori, z, tv, z, rv)
    return {"b": b, "x": x, "tvel": tv, "rvel": rv, "pos": npos, "ori": nori}


def _gpu_step0(cfg, pos, ori):
    from rigidfibers_b200 import Simulation
    sim = Simulation(cfg, pos, ori)
    sim.assembleSystem()
    sim.solveSystem()
    x = sim.solution()
    sim.updateVelocities()
    tv, rv = sim.velocities()
    sim.updateFibers(True)
    p1, o1 = sim.state()
    st = sim.stats()
    sim.close()
    return {"x": x, "tvel": tv, "rvel": rv, "pos": p1, "ori": o1, "iterations": st["iterations"],
            "relres": st["relative_residual"]}


def _rel_errors(got, ref):
    out = {}
    for k, name in (("x", "forces"), ("tvel", "tvel"), ("rvel", "rvel"), ("pos", "pos"), ("ori", "ori")):
        a = np.asarray(got[k], np.float64).reshape(-1)
        r = np.asarray(ref[k], np.float64).reshape(-1)
        out[name] = float(np.abs(a - r).max() / max(np.abs(r).max(), 1e-30))
    out["max"] = max(out.values())
    return out


def _mem_available_gb():
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def error_vs_fp64(args, precision):
    """Errors of whole time steps against the FP64 reference at the benchmark
    configurations (max |ours - FP64| / max |FP64| per field, step 0 from the
    seeded layout): N fibers of the headline workload for the mixed and the
    plain FP32 path, and N=direct_fibers analytical fibers for GMRES and the
    direct solver."""
    from rigidfibers_b200 import Config
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    out = {"method": "step 0 from the seeded layout; FP64 reference = the oracle's FP64 assembly and velocities on "
                     "the host cores, FP64 LU solve on the GPU (torch.linalg.solve) as the checker; "
                     "max |ours - FP64| / max |FP64| per field"}
    N = args.fibers
    need = 2.2 * (15 * N) ** 2 * 8 / 1e9
    if _mem_available_gb() < need:
        out["headline"] = {"unavailable": "host memory: %.0f GB available, %.0f GB needed" %
                                          (_mem_available_gb(), need)}
    else:
        pos, ori = workload(args)
        ours = {precision: _gpu_step0(Config(precision=precision, refinement_restart=args.mixed_restart), pos, ori),
                "fp32": _gpu_step0(Config(precision="fp32"), pos, ori),
                "direct": _gpu_step0(Config(solver="direct"), pos, ori)}
        ref = fp64_reference_step(pos, ori)
        out["headline"] = {"fibers": N, "integration": "numerical"}
        for k, g in ours.items():
            out["headline"][k] = _rel_errors(g, ref)
            out["headline"][k]["gmres_iterations"] = g["iterations"]
    if args.direct_fibers > 0:
        n = args.direct_fibers
        radius = 14.0 * (n / 2000.0) ** (1.0 / 3.0)
        pos, ori = sphere_layout(n, radius, 0.2, seed=layout_seed(2, n))
        ours = {s: _gpu_step0(Config(solver=s, integration="analytical"), pos, ori) for s in ("gmres", "direct")}
        ref = fp64_reference_step(pos, ori, analytical=True)
        out["thesis_scale"] = {"fibers": n, "integration": "analytical"}
        for k, g in ours.items():
            out["thesis_scale"][k] = _rel_errors(g, ref)
    return out


def serve_ensemble(args, dist, pack_fibers=None, max_active=None):
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
    slots = args.serve_max_active if max_active is None else max_active
    ids = []
    with Server(max_active=slots, use_cuda_graphs=args.serve_graphs, pack_max_fibers=pack) as srv:
        t0 = time.perf_counter()
        due = t0
        for r, (p, o), c, g in zip(reqs, layouts, cfgs, gaps):
            due += g
            delay = due - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(c, p, o, r["nsteps"]))
        srv.drain()
        wall = time.perf_counter() - t0
        st = srv.stats()
        # per-step latencies by request size (the mix spans 16..1000 fibers, so
        # the overall tail is mostly the large requests' steps)
        by_size = {}
        for r, rid in zip(reqs, ids):
            lo = next(b for b in (512, 256, 128, 64, 16) if r["n"] >= b)
            by_size.setdefault(lo, []).extend(srv.step_times(rid).tolist())
        size_classes = {"%d-%d" % (lo, {16: 63, 64: 127, 128: 255, 256: 511, 512: 1000}[lo]):
                        {"steps": len(v), "p50_step_ms": float(np.percentile(v, 50)),
                         "p99_step_ms": float(np.percentile(v, 99))}
                        for lo, v in sorted(by_size.items()) if v}
    dist.barrier()
    wall_max = dist.max(wall)
    fiber_steps = dist.sum(st["fiber_steps"])
    return {"p50_step_ms": st["p50_step_ms"], "p99_step_ms": st["p99_step_ms"],
            "p50_setup_ms": st["p50_setup_ms"], "p99_setup_ms": st["p99_setup_ms"],
            "fiber_steps_per_s": fiber_steps / wall_max, "requests": len(reqs) * dist.world,
            "completed": int(dist.sum(st["completed"])), "failed": int(dist.sum(st["failed"])),
            "steps": int(dist.sum(st["steps"])), "wall_s": wall_max, "arrival_rate_per_s": args.serve_rate,
            "max_active": slots, "peak_active": st["peak_active"],
            "cuda_graph_mode": args.serve_graphs, "pack_max_fibers": pack,
            **({"pack_steps": st["pack_steps"], "pack_p50_ms": st["pack_p50_ms"], "pack_p99_ms": st["pack_p99_ms"],
                "pack_max_ms": st["pack_max_ms"], "pack_mean_members": st["pack_mean_members"]} if pack else {}),
            "by_size": size_classes,
            "peak_device_bytes": st["peak_bytes"], "storage": "mixed_bf16",
            "workload": "N log-uniform in [16, 1000], eps 0.01 or 0.005, 5-50 steps, Poisson arrivals; latency = "
                        "host wall time of one step while others run; setup = admission to ready (handle created, "
                        "step graphs built)"}


def direct_leg(args, n=None, integration="analytical", solvers=("direct", "gmres")):
    """A direct-solver configuration: by default the thesis scale (N=2000
    fibers in a radius-14 sphere, analytical integration), one step solved by
    the blocked LU (in place of MAGMA's sgesv) and by GMRES on the same system;
    with n and integration given, that layout (the precision configuration:
    N=4000, radius 18, numerical).  LU rate = 2/3 R^3 flops over the solve time
    (factorisation, triangular solves and FP64 refinement)."""
    from rigidfibers_b200 import Config, Simulation
    from rigidfibers_b200.generate import layout_seed, sphere_layout
    if n is None:
        n = args.direct_fibers
        radius = 14.0 * (n / 2000.0) ** (1.0 / 3.0)
        pos, ori = sphere_layout(n, radius, 0.2, seed=layout_seed(2, n))
    else:
        radius = 18.0 * (n / 4000.0) ** (1.0 / 3.0)
        pos, ori = workload_layout(n, radius)
    out = {"fibers": n, "radius": radius, "integration": integration}
    for solver in solvers:
        sim = Simulation(Config(solver=solver, integration=integration), pos, ori)
        sim.step(0)                      # warm-up (first-touch of the kernels)
        sim.autotune()
        ck = sim.checkpoint()
        sim.step(1)                      # the timed step: the stage times come from rf_step
        st = sim.stats()
        sim.restore(ck)
        sim.close()
        R = 15 * n
        leg = {"ms_solve": st["ms_solve_system"], "ms_assemble": st["ms_assemble_system"],
               "relative_residual": st["relative_residual"], "iterations": st["iterations"],
               "refinements": st["refinement_steps"]}
        if solver == "direct":
            leg["tflops"] = (2.0 / 3.0) * R ** 3 / (st["ms_solve_system"] / 1e3) / 1e12
            leg["row_exchanges"] = bool(st["pivoted"])
            leg["max_multiplier"] = st["max_multiplier"]
        out[solver] = leg
    return out


def _plain(args, dist, total_fiber_steps, cfg):
    r = time_path(args, dist, cfg, *workload(args))
    ms = dist.max(r["ms"])
    return {"value": total_fiber_steps / (ms / 1000.0), "ms_per_step": ms / args.steps,
            "gmres_restart": cfg.gmres_restart,
            "stage_ms_per_step": {k: v / args.steps for k, v in r["stage"].items()},
            "gmres_iterations_per_step": r["iters"] / args.steps}, r


def run_ours(args, dist):
    import torch

    from rigidfibers_b200 import Config

    torch.cuda.set_device(dist.local)
    pos, ori = workload(args)
    N = args.fibers
    R = 15 * N
    precision = "mixed_fp16" if args.precision == "auto" else args.precision
    cfg = Config(precision=precision, refinement_restart=args.mixed_restart)
    if precision == "matrix_free":
        # the FP32 path's GMRES with the mixed path's restart length (GMRES(10)
        # stalls on the largest systems)
        cfg = Config(precision=precision, gmres_restart=args.mixed_restart or 10)
    head = time_path(args, dist, cfg, pos, ori, clocks=Clocks(dist.local))
    ms_max, total_fiber_steps, value = whole_job_rate(dist, head["ms"], N * args.steps)
    e2e_s, e2e_iters, ck_bytes = e2e_path(args, dist, cfg, pos, ori)
    e2e_value = total_fiber_steps / e2e_s

    comparison = matched = None
    if precision not in ("fp32", "matrix_free") and not args.no_fp32_path:
        comparison, plain = _plain(args, dist, total_fiber_steps, Config(precision="fp32"))
        # the mixed path runs mixed_restart Arnoldi steps between corrections;
        # FP32 GMRES with the same restart length separates precision from restart
        matched, _ = _plain(args, dist, total_fiber_steps,
                            Config(precision="fp32", gmres_restart=args.mixed_restart or 10))

    hbm, peak_kind = peaks()
    mvn = max(head["mv_launches"], 1)
    mv_avg_ms = head["mv_ms"] / mvn
    mfree = precision == "matrix_free"
    if precision == "fp32":
        kernel = "k_gemv_cm_f32 (dense FP32 column-major matvec, GMRES)"
        bytes_per_matvec = 4.0 * R * R
    elif mfree:
        kernel = ("k_assemble_pairs<5,24,apply> + k_sum_parts + k_struct_finalize (matrix-free product: the pair "
                  "blocks recomputed and applied, nothing read but the fiber state and x)")
        bytes_per_matvec = 0.0
    else:
        kernel = ("k_struct_z16_bulk<5> + k_sum_parts + k_struct_finalize (16-bit structured matvec, "
                  "TMA bulk-copy pipeline, GMRES)")
        bytes_per_matvec = 2.0 * 150 * N * (N - 1) / 2
    achieved = bytes_per_matvec / (mv_avg_ms / 1000.0) / 1e9 if head["mv_launches"] else None
    # DRAM traffic per launch from one ncu capture of the same kernel at N=1500
    # (dram__bytes_read.sum 347.6 MB + dram__bytes_write.sum 9.8 MB for 1124250
    # unordered pairs: 304-byte records for 300 algorithmic bytes, x, partial
    # rows), scaled by the pairs one launch processes; not captured for the
    # dense FP32 kernel
    traffic = 357.4e6 / (1500 * 1499 / 2) * (N * (N - 1) / 2) if precision not in ("fp32", "matrix_free") else None
    if precision == "fp32":
        # one ncu capture of k_gemv_cm_f32 at N=1000: dram__bytes_read.sum 900.6 MB
        # + dram__bytes_write.sum 5.0 MB for R^2 x 4 B = 900.0 MB, scaled by R^2
        traffic = (900.6e6 + 5.0e6) / (4.0 * 15000 ** 2) * bytes_per_matvec
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None, "traffic": traffic, "peak_kind": peak_kind,
            "kernel": kernel,
            "traffic_source": None if traffic is None else ("ncu capture at N=1000 scaled by R^2" if precision == "fp32"
                                                            else "ncu capture at N=1500 scaled by pairs"),
            "algorithmic_bytes_per_launch": bytes_per_matvec, "avg_launch_ms": mv_avg_ms,
            "launches": head["mv_launches"], "share_of_step_time": head["mv_ms"] / head["ms"] if head["ms"] else None,
            "measured_in": "a profiled pass of the same K steps after the timed ones (CUDA events around each matvec "
                           "launch on the handle's stream; per-launch events rule out graph replay)"}
    if mfree:
        # the product recomputes every pair block: FP32 issue-bound like the assembly
        fl = ASM_EXEC_FLOPS_PER_PAIR * N * (N - 1) / 2
        ach = fl / (mv_avg_ms / 1000.0) / 1e12 if head["mv_launches"] else None
        roof.update({"bound": "fp32", "achieved": ach, "peak": NOMINAL_FP32_TFLOPS, "unit": "TFLOP/s",
                     "frac": ach / NOMINAL_FP32_TFLOPS if ach else None, "peak_kind": "nominal FP32 SIMT",
                     "algorithmic_flops_per_launch": fl})
    out = {
        "metric": METRIC, "value": value, "unit": "fiber-steps/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if precision in ("fp32", "matrix_free") else
                 "%s storage, f32 accumulate, f64 refinement" % precision[6:],
        "data": "synthetic",
        "config": {"workload": workload_name(args), "fibers": N, "radius": args.radius, "precision": precision,
                   "parallelism": "replicas x%d" % dist.world,
                   "l2": "inputs larger than L2: the operator (%.1f GB) is re-assembled and re-read every step"
                         % (head["device_bytes"] / 1e9)},
        "roofline": roof, "clocks": head["clocks"],
        "e2e": {"value": e2e_value, "unit": "fiber-steps/s", "h2d_bytes_per_step": ck_bytes,
                "d2h_bytes_per_step": ck_bytes, "gmres_iterations_per_step": e2e_iters,
                "timing": "host wall clock, max over ranks; the same K steps as the device-timed pass, with the "
                          "state in pinned host memory between steps (rf_checkpoint_load, rf_step, "
                          "rf_checkpoint_save)"},
        "gpu_launches": head["launches"],
        "stage_ms_per_step": {k: v / args.steps for k, v in head["stage"].items()},
        "gmres_iterations_per_step": head["iters"] / args.steps,
        "refinements_per_step": head["refinements"] / args.steps,
        "graph_replays_per_step": head["graph_replays"] / args.steps,
        "max_relative_residual": head["relres"],
        "matvec_variant": head["autotune"]["matvec_variant"],
        "autotune": {k: head["autotune"][k] for k in ("asm_variant", "asm_ms", "matvec_variant", "matvec_ms")},
    }
    if args.direct_fibers > 0 and dist.rank == 0:
        out["direct_solver"] = direct_leg(args)
        if args.direct_large_fibers > 0:
            out["direct_solver_precision_config"] = direct_leg(args, args.direct_large_fibers, "numerical", ("direct",))
    head["steps"] = args.steps
    if not mfree:
        out["kernels"] = kernel_rooflines(N, head, hbm, precision != "fp32", out.get("direct_solver"))
    if dist.rank == 0 and not args.no_cpu_baseline:
        res = cpu_steps(pos, ori, 1, untimed=0)
        out["cpu_baseline"] = {"value": res["value"], "unit": "fiber-steps/s", "cores": res["cores"],
                               "kind": CPU_KIND, "seconds_per_step": res["seconds_per_step"],
                               "gmres_iterations": res["gmres_iterations_per_step"],
                               "sample": "%s; one full time step (step 0) of the N=%d workload" % (CPU_WHAT, N)}
    if dist.rank == 0 and not args.no_error_leg:
        out["error_vs_fp64"] = error_vs_fp64(args, precision)
    if comparison:
        out["fp32_path"] = comparison
        out["fp32_restart_matched"] = matched
    if args.serve_requests > 0:
        if args.serve_compare:
            cp, ca = (int(v) for v in args.serve_compare.split(","))
            out["serving_compare"] = serve_ensemble(args, dist, cp, ca)
        out["serving"] = serve_ensemble(args, dist)
    # the headline figures once more, compact, at the end of the line
    summ = {"value": value, "e2e": e2e_value}
    if comparison:
        summ["speedup_vs_fp32_gmres10"] = value / comparison["value"]
        summ["speedup_vs_fp32_restart_matched"] = value / matched["value"]
    err = (out.get("error_vs_fp64") or {}).get("headline") or {}
    for k in (precision, "fp32"):
        if k in err:
            summ["error_vs_fp64_%s_N%d" % (k, N)] = err[k]["max"]
    if "serving" in out:
        summ.update(serving_p50_ms=out["serving"]["p50_step_ms"], serving_p99_ms=out["serving"]["p99_step_ms"],
                    serving_fiber_steps_per_s=out["serving"]["fiber_steps_per_s"])
    if "cpu_baseline" in out:
        summ["cpu_baseline"] = out["cpu_baseline"]["value"]
    out["summary"] = summ
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
        if args.serve_compare:
            cp, ca = (int(v) for v in args.serve_compare.split(","))
            out["serving_compare"] = serve_ensemble(args, dist, cp, ca)
    if "direct" in legs and dist.rank == 0:
        out["direct_solver"] = direct_leg(args)
    if "error" in legs and dist.rank == 0:
        out["error_vs_fp64"] = error_vs_fp64(args, "mixed_fp16" if args.precision == "auto" else args.precision)
    if "cpu" in legs and dist.rank == 0:
        pos, ori = workload(args)
        out["cpu"] = cpu_steps(pos, ori, args.steps, untimed=1, cap_s=args.reference_cap_s)
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
