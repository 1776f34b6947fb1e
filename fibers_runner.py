#!/usr/bin/env python3
"""Run, validate and benchmark the rigid-fiber simulation on a B200.

Same command line as the reference's runner (fibers_runner.py:17-162,
runner/cuda_runner.py), in Python 3, over the CUDA library (no per-run
recompilation: N, M, Q, the solver and the integration are runtime values):

    fibers_runner.py cuda run       (--magma|--gmres|--bicgstab) (--numerical|--analytical)
                                    (--D1|--D2|--D3) configuration_file fibers_file
    fibers_runner.py cuda validate  ... configuration_file fibers_file [--reference DIR]
    fibers_runner.py cuda benchmark [--max_rse F] ... configuration_file [--sizes 2000,1900,...]

--magma selects the direct solver (the reference called MAGMA's sgesv).
--D1/--D2/--D3 chose a CUDA thread mapping of the reference's assembly; they
are accepted for compatibility and all run the same pair-tile kernel.
Extra options of this build: --precision {fp32,mixed_fp16,mixed_bf16,matrix_free,
mixed_fp16_recompute,mixed_bf16_recompute},
--velocity-integration {same,numerical,analytical}, --output DIR.

Outputs (same formats as the reference):
  run       XcT_res_%05d.out / TcR_res_%05d.out every STATE_SAVE_INTERVAL /
            VELOCITY_SAVE_INTERVAL steps (src/simulation.cu:530-604)
  validate  {t}_{BVec,XVec,TRANSVel,ROTVel,POS,ORIENT}.out dumps (F16.8, one
            value per line; fortran/fibers.f95:205-303), compared field by field
            against reference vectors with pass/fail tolerances (the reference's
            tools/validate.py only prints the differences)
  benchmark performance.out per run (name,time) and results.csv (tab-separated,
            mean and sample deviation per step name; runner/cuda_runner.py:217-339)
"""
import argparse
import csv
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from rigidfibers_b200 import formats as F  # noqa: E402

FIELDS = ["BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT"]
STEP_NAMES = ["assemble_system", "solve_system", "update_velocities", "update_fibers"]


def _solver(args):
    return "direct" if args.magma else ("bicgstab" if args.bicgstab else "gmres")


def _integration(args):
    return "analytical" if args.analytical else "numerical"


def make_config(params, args):
    from rigidfibers_b200 import Config
    return Config.from_ini(params, solver=_solver(args), integration=_integration(args),
                           precision=args.precision, velocity_integration=args.velocity_integration)


def _out(args, name):
    os.makedirs(args.output, exist_ok=True)
    return os.path.join(args.output, name)


# ---------------------------------------------------------------------------
# run (runner/cuda_runner.py:154-161 + src/main.cu:85-99)
# ---------------------------------------------------------------------------
def run(args):
    from rigidfibers_b200 import Simulation
    params = F.read_config(args.configuration_file)
    pos, ori = F.read_fibers(args.fibers_file)
    sim = Simulation(make_config(params, args), pos, ori)
    steps = params["NUMBER_OF_TIMESTEPS"]
    ssi, vsi = params["STATE_SAVE_INTERVAL"], params["VELOCITY_SAVE_INTERVAL"]
    log = open(args.json_log, "w") if getattr(args, "json_log", None) else None
    t0 = time.time()
    for t in range(steps):
        sim.step(t)
        if log is not None:
            log.write(step_record(t, sim.N, sim.stats()) + "\n")
            log.flush()
        if ssi > 0 and t % ssi == 0:
            p, o = sim.state()
            F.write_fibers(_out(args, "XcT_res_%05d.out" % (t + 1)), p, o)
        if vsi > 0 and t % vsi == 0:
            tv, rv = sim.velocities()
            F.write_fibers(_out(args, "TcR_res_%05d.out" % (t + 1)), tv, rv)
        if args.verbose:
            st = sim.stats()
            print("[GPU] step %d: %s, %d iterations, residual %.2e" % (
                t, ", ".join("%s %.3f ms" % (n, st["ms_" + n]) for n in STEP_NAMES), st["iterations"],
                st["relative_residual"]))
    if log is not None:
        log.close()
    print("**************************************************")
    print("  %d fibers, %d steps in %.3f s" % (sim.N, steps, time.time() - t0))
    return 0


def step_record(t, n_fibers, st):
    """One JSON line per time step: the per-stage device times and the solver
    counters of that step (the numbers the reference prints per step under
    --verbose, src/main.cu:85-99, as machine-readable records)."""
    rec = {"step": t, "fibers": n_fibers}
    rec.update({k: (round(v, 6) if isinstance(v, float) else v) for k, v in st.items()})
    # a step run as one CUDA graph reports its total only (stage times 0)
    rec["ms_step"] = round(st["ms_step"] if st.get("ms_step", 0.0) > 0 else sum(st["ms_" + n] for n in STEP_NAMES), 6)
    return json.dumps(rec, sort_keys=True)


# ---------------------------------------------------------------------------
# validate (runner/cuda_runner.py:163-215)
# ---------------------------------------------------------------------------
def reference_vectors(args, pos, ori):
    """{(t, field): values} from --reference DIR ({t}_{field}.ref files), or
    the reference's packed 100-fiber golden files when the layout is that one."""
    if args.reference:
        out = {}
        for t in range(2):
            for f in FIELDS:
                p = os.path.join(args.reference, "%d_%s.ref" % (t, f))
                if os.path.exists(p):
                    out[(t, f)] = F.read_column(p)
        return out
    golden = os.path.join(ROOT, "tests", "golden", "ref100.npz")
    g = np.load(golden)
    if pos.shape != g["positions"].shape or np.abs(pos - g["positions"]).max() > 1e-12 or \
            np.abs(ori - g["orientations"]).max() > 1e-12:
        raise SystemExit("validate: no reference vectors for this layout (give --reference DIR)")
    var = ("analytic_" if args.analytical else "numeric_") + ("gmres" if _solver(args) == "gmres" else "direct")
    return {(t, f): g["%s/%d_%s" % (var, t, f)] for t in range(2) for f in FIELDS}


def validate(args):
    from rigidfibers_b200 import Simulation
    params = F.read_config(args.configuration_file)
    params["NUMBER_OF_TIMESTEPS"] = 2   # the reference vectors hold two steps
    pos, ori = F.read_fibers(args.fibers_file)
    refs = reference_vectors(args, pos, ori)
    sim = Simulation(make_config(params, args), pos, ori)
    # tolerances relative to each field's largest magnitude; Krylov solutions
    # differ from a direct one by up to the solver tolerance
    tol = {"gmres": 1e-5, "direct": 1e-5, "bicgstab": 5e-5}[_solver(args)]
    if args.precision.startswith("mixed"):
        tol = 1e-4   # the 16-bit operator's bound; the matrix-free mode keeps the plain path's
    failed = []
    for t in range(2):
        sim.assembleSystem()
        _, b = sim.system(with_matrix=False)
        sim.solveSystem()
        x = sim.solution()
        sim.updateVelocities()
        tv, rv = sim.velocities()
        sim.updateFibers(t == 0)
        p, o = sim.state()
        dumps = {"BVec": b, "XVec": x, "TRANSVel": tv, "ROTVel": rv, "POS": p, "ORIENT": o}
        for f in FIELDS:
            F.write_column(_out(args, "%d_%s.out" % (t, f)), dumps[f])
            if (t, f) not in refs:
                continue
            ref = np.asarray(refs[(t, f)], np.float64).reshape(-1)
            cur = np.asarray(dumps[f], np.float64).reshape(-1)
            if ref.shape != cur.shape:
                print("  [FAIL] %d_%s: shape %s vs reference %s" % (t, f, cur.shape, ref.shape))
                failed.append((t, f))
                continue
            diff = np.abs(cur - ref)
            rel = diff.max() / max(np.abs(ref).max(), 1e-30)
            ok = rel <= tol
            print("  [%s] %d_%-8s max |d| %.3e  mean |d| %.3e  relative %.2e (tolerance %.0e)" % (
                "PASS" if ok else "FAIL", t, f, diff.max(), diff.mean(), rel, tol))
            if not ok:
                failed.append((t, f))
    print("**************************************************")
    if failed:
        print("  validation FAILED: %s" % ", ".join("%d_%s" % k for k in failed))
        return 1
    print("  validation passed")
    return 0


# ---------------------------------------------------------------------------
# benchmark (runner/cuda_runner.py:217-339)
# ---------------------------------------------------------------------------
def benchmark(args):
    from rigidfibers_b200 import Simulation
    from rigidfibers_b200.generate import grown_sphere_layout, layout_seed
    params = F.read_config(args.configuration_file)
    sizes = [int(s) for s in args.sizes.split(",")] if args.sizes else list(range(2000, 0, -100))
    results = {}
    for idx, n in enumerate(sizes):
        print("  [BENCHMARK]   : %d fibers (%d/%d)" % (n, idx + 1, len(sizes)))
        runs = []
        want = 4
        rse = float("inf")
        rep = 0
        while rse > args.max_rse:
            while len(runs) < want:
                pos, ori = grown_sphere_layout(n, args.min_distance, seed=layout_seed(100 + rep, n))
                rep += 1
                sim = Simulation(make_config(params, args), pos, ori, allow_noconv=True)
                # per-stage times (performance.out) need the stages launched one by one:
                # CUDA graphs for the restart cycles only
                sim.set_cuda_graphs(2)
                acc = {k: [] for k in STEP_NAMES}
                for t in range(params["NUMBER_OF_TIMESTEPS"]):
                    sim.step(t)
                    if t == 0:
                        continue   # the first step is the warm-up (src/performance.cc:73-78)
                    st = sim.stats()
                    for k in STEP_NAMES:
                        acc[k].append(st["ms_" + k] / 1000.0)
                sim.close()
                run_ = {k: float(np.mean(v)) if v else 0.0 for k, v in acc.items()}
                run_["total"] = sum(run_[k] for k in STEP_NAMES)
                with open(_out(args, "performance.out"), "w") as fh:
                    fh.write("name,time\n")
                    for k in STEP_NAMES:
                        fh.write("%s,%.8f\n" % (k, run_[k]))
                runs.append(run_)
            totals = [r["total"] for r in runs]
            mean = float(np.mean(totals))
            sd = float(np.std(totals, ddof=1)) if len(totals) > 1 else 0.0
            rse = (sd / math.sqrt(len(totals))) / mean if mean > 0 else 0.0
            if rse > args.max_rse:
                want = len(runs) * 2
                print("                : Relative Standard Error: %d%% - increasing iterations to %d"
                      % (round(rse * 100), want))
        row = {}
        for k in STEP_NAMES + ["total"]:
            vals = [r[k] for r in runs]
            row[k] = float(np.mean(vals))
            row[k + "_std"] = float(np.std(vals, ddof=1)) if len(vals) > 1 else 0.0
        results[n] = row
    keys = sorted(next(iter(results.values())).keys())
    with open(_out(args, "results.csv"), "w", newline="") as fh:
        w = csv.writer(fh, dialect="excel-tab")
        w.writerow(["X"] + keys)
        print("**************************************************")
        print("Benchmark:")
        print("  " + "\t".join(["X"] + keys))
        for n in sorted(results):
            r = [n] + [results[n][k] for k in keys]
            w.writerow(r)
            print("  " + "\t".join(str(v) for v in r))
    print("**************************************************")
    return 0


def fortran_unavailable(args):
    print("the fortran platform is the reference's own CPU program (gfortran + OpenBLAS); it is not part of "
          "this build -- use the cuda platform", file=sys.stderr)
    return 2


def build_parser():
    ap = argparse.ArgumentParser(description="Helper program for running, validating and benchmarking the rigid "
                                             "fibers simulation")
    ap.add_argument("--verbose", action="store_true", help="be verbose")
    plat = ap.add_subparsers(title="supported platforms", dest="platform")
    plat.required = True
    pc = plat.add_parser("cuda", help="CUDA implementation (B200)")
    cmds = pc.add_subparsers(title="supported commands", dest="command")
    cmds.required = True
    for name, fn, fibers in (("run", run, True), ("validate", validate, True), ("benchmark", benchmark, False)):
        p = cmds.add_parser(name, help="%s the simulation" % name)
        p.set_defaults(func=fn)
        p.add_argument("configuration_file", type=str, help="the configuration file")
        if fibers:
            p.add_argument("fibers_file", type=str, help="the file containing the initial positions and orientations")
        g = p.add_argument_group("supported solvers").add_mutually_exclusive_group(required=True)
        g.add_argument("--magma", action="store_true")
        g.add_argument("--gmres", action="store_true")
        g.add_argument("--bicgstab", action="store_true")
        g = p.add_argument_group("supported algorithms").add_mutually_exclusive_group(required=True)
        g.add_argument("--numerical", action="store_true")
        g.add_argument("--analytical", action="store_true")
        g = p.add_argument_group("supported parallization dimensions").add_mutually_exclusive_group(required=True)
        g.add_argument("--D1", action="store_true")
        g.add_argument("--D2", action="store_true")
        g.add_argument("--D3", action="store_true")
        p.add_argument("--precision", default="fp32",
                       choices=["fp32", "mixed_fp16", "mixed_bf16", "matrix_free", "mixed_fp16_recompute",
                                "mixed_bf16_recompute"])
        p.add_argument("--velocity-integration", default="same", choices=["same", "numerical", "analytical"])
        p.add_argument("--output", default=".", help="directory for the output files")
        if name == "run":
            p.add_argument("--json-log", default=None, help="write one JSON line of step statistics per time step")
        if name == "validate":
            p.add_argument("--reference", default=None, help="directory of {t}_{field}.ref reference vectors")
        if name == "benchmark":
            p.add_argument("--max_rse", type=float, default=0.2,
                           help="the maximum relative standard error (default: 0.2)")
            p.add_argument("--sizes", default=None, help="comma-separated fiber counts (default 2000..100 step 100)")
            p.add_argument("--min-distance", type=float, default=0.2)
    pf = plat.add_parser("fortran", help="the reference's OpenMP Fortran program (not part of this build)")
    pf.add_argument("rest", nargs=argparse.REMAINDER)
    pf.set_defaults(func=fortran_unavailable)
    return ap


def main(argv=None):
    args = build_parser().parse_args(argv)
    return args.func(args)


if __name__ == "__main__":
    sys.exit(main())
