"""fibers_runner.py: the reference's command line (fibers_runner.py:17-162)."""
import json
import os

import numpy as np
import pytest

import fibers_runner as FR
from rigidfibers_b200 import formats as F


def write_inputs(tmp_path, golden, steps=2):
    conf = json.loads(str(golden["config_json"]))
    conf["RUN"]["number_of_timesteps"] = str(steps)
    ini = tmp_path / "config.ini"
    with open(ini, "w") as fh:
        for sec, kv in conf.items():
            fh.write("[%s]\n" % sec)
            for k, v in kv.items():
                fh.write("%s=%s\n" % (k.upper(), v))
    fib = tmp_path / "XcT_ref100.in"
    F.write_fibers(str(fib), golden["positions"], golden["orientations"], fmt="%.16f")
    return str(ini), str(fib)


def test_parser_accepts_reference_command_lines():
    p = FR.build_parser()
    a = p.parse_args(["cuda", "run", "--gmres", "--numerical", "--D2", "c.ini", "f.in"])
    assert a.func is FR.run and a.gmres and a.numerical
    a = p.parse_args(["cuda", "validate", "--magma", "--analytical", "--D1", "c.ini", "f.in"])
    assert FR._solver(a) == "direct" and FR._integration(a) == "analytical"
    a = p.parse_args(["cuda", "benchmark", "--max_rse", "0.1", "--bicgstab", "--numerical", "--D3", "c.ini"])
    assert a.max_rse == 0.1 and FR._solver(a) == "bicgstab"
    with pytest.raises(SystemExit):
        p.parse_args(["cuda", "run", "--gmres", "--bicgstab", "--numerical", "--D2", "c.ini", "f.in"])
    with pytest.raises(SystemExit):
        p.parse_args(["cuda", "run", "--gmres", "--D2", "c.ini", "f.in"])


def test_step_record_is_one_json_object():
    st = {"iterations": 7, "restarts": 0, "refinement_steps": 1, "relative_residual": 3.5e-7,
          "ms_assemble_system": 1.25, "ms_solve_system": 2.5, "ms_update_velocities": 0.25, "ms_update_fibers": 0.0,
          "device_bytes": 1 << 20, "kernel_launches": 40, "graph_replays": 2, "factorizations": 0}
    line = FR.step_record(3, 100, st)
    assert "\n" not in line
    rec = json.loads(line)
    assert rec["step"] == 3 and rec["fibers"] == 100 and rec["iterations"] == 7
    assert rec["ms_step"] == 4.0
    a = FR.build_parser().parse_args(["cuda", "run", "--gmres", "--numerical", "--D2", "c.ini", "f.in",
                                      "--json-log", "s.jsonl"])
    assert a.json_log == "s.jsonl"


def test_fortran_platform_is_reported_unavailable():
    assert FR.main(["fortran", "run", "--direct", "--numerical", "c.ini", "f.in"]) == 2


@pytest.mark.gpu
def test_run_writes_reference_state_files(tmp_path, golden):
    ini, fib = write_inputs(tmp_path, golden, steps=2)
    out = tmp_path / "out"
    assert FR.main(["cuda", "run", "--gmres", "--numerical", "--D2", ini, fib, "--output", str(out)]) == 0
    p, o = F.read_fibers(str(out / "XcT_res_00002.out"))
    assert np.abs(p.reshape(-1) - golden["numeric_gmres/1_POS"]).max() < 1e-5
    assert np.abs(o.reshape(-1) - golden["numeric_gmres/1_ORIENT"]).max() < 1e-5
    tv, rv = F.read_fibers(str(out / "TcR_res_00001.out"))
    assert np.abs(tv.reshape(-1) - golden["numeric_gmres/0_TRANSVel"]).max() < 1e-4


@pytest.mark.gpu
def test_run_writes_json_step_log(tmp_path, golden):
    ini, fib = write_inputs(tmp_path, golden, steps=3)
    log = tmp_path / "steps.jsonl"
    assert FR.main(["cuda", "run", "--gmres", "--numerical", "--D2", ini, fib, "--output", str(tmp_path / "o"),
                    "--json-log", str(log)]) == 0
    recs = [json.loads(line) for line in open(str(log))]
    assert [r["step"] for r in recs] == [0, 1, 2]
    for r in recs:
        assert r["fibers"] == 100 and r["iterations"] > 0 and r["relative_residual"] < 1e-5
        assert r["ms_step"] > 0 and r["kernel_launches"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [["--gmres", "--numerical"], ["--gmres", "--analytical"], ["--bicgstab", "--numerical"],
                                   ["--gmres", "--numerical", "--precision", "mixed_fp16"],
                                   ["--bicgstab", "--numerical", "--precision", "mixed_fp16"],
                                   ["--gmres", "--numerical", "--precision", "matrix_free"],
                                   ["--bicgstab", "--numerical", "--precision", "mixed_bf16_recompute"]])
def test_validate_passes_against_golden(tmp_path, golden, flags):
    ini, fib = write_inputs(tmp_path, golden)
    out = tmp_path / "v"
    rc = FR.main(["cuda", "validate"] + flags[:2] + ["--D2", ini, fib, "--output", str(out)] + flags[2:])
    assert rc == 0
    assert os.path.exists(str(out / "1_XVec.out"))


@pytest.mark.gpu
def test_validate_fails_on_wrong_reference(tmp_path, golden):
    ini, fib = write_inputs(tmp_path, golden)
    ref = tmp_path / "ref"
    ref.mkdir()
    F.write_column(str(ref / "0_BVec.ref"), golden["numeric_gmres/0_BVec"] * 1.01)
    rc = FR.main(["cuda", "validate", "--gmres", "--numerical", "--D2", ini, fib, "--output", str(tmp_path / "v"),
                  "--reference", str(ref)])
    assert rc == 1


@pytest.mark.gpu
def test_benchmark_writes_results(tmp_path, golden):
    ini, _ = write_inputs(tmp_path, golden, steps=3)
    out = tmp_path / "b"
    assert FR.main(["cuda", "benchmark", "--gmres", "--numerical", "--D2", ini, "--sizes", "40,20",
                    "--max_rse", "10", "--output", str(out)]) == 0
    rows = open(str(out / "results.csv")).read().splitlines()
    assert rows[0].split("\t")[0] == "X" and "total" in rows[0].split("\t")
    assert [r.split("\t")[0] for r in rows[1:]] == ["20", "40"]
