"""bench.py's multi-GPU plumbing on the host: world_size-2 gloo ranks.  The
data path has no collective (independent replicas); only the whole-job rate
(slowest rank's time, units of all ranks) and the barrier cross ranks, and the
reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(world, backend="gloo")
    d.barrier()
    ms, total, rate = bench.whole_job_rate(d, 10.0 * (rank + 1), 100 * (rank + 1))
    d.barrier()
    d.close()
    with open(os.path.join(out, "r%d.json" % rank), "w") as fh:
        json.dump({"ms": ms, "total": total, "rate": rate}, fh)


def test_whole_job_rate_over_two_gloo_ranks(tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        got = json.load(open(tmp_path / ("r%d.json" % r)))
        assert got["ms"] == 20.0 and got["total"] == 300.0
        assert abs(got["rate"] - 300.0 / 0.020) < 1e-6


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
