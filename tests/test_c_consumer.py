"""A plain C program compiled against include/rigidfibers.h and linked with
librigidfibers.so: the binding a C or C++ host of the reference's step seam
(src/simulation.h:38-97) would write.  Compiling and linking needs no GPU;
running it on the reference's 100-fiber golden layout for two steps must
reproduce the golden positions and orientations (1e-5 relative, the plain
FP32 path's tolerance)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_consumer", "golden_steps.c")
LIBDIR = os.path.join(ROOT, "rigidfibers_b200")


def _cc():
    for c in ("/usr/bin/gcc", "gcc", "cc"):
        if shutil.which(c):
            return c
    pytest.skip("no C compiler")


def build(tmp_path):
    exe = str(tmp_path / "golden_steps")
    cmd = [_cc(), "-std=c99", "-Wall", "-Werror", "-O2", SRC, "-I", os.path.join(ROOT, "include"), "-L", LIBDIR,
           "-lrigidfibers", "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_c_consumer_compiles_and_links(tmp_path):
    exe = build(tmp_path)
    assert os.access(exe, os.X_OK)
    # the program checks its arguments before touching the library or the device
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("solver,variant", [("gmres", "numeric_gmres"), ("direct", "numeric_direct")])
def test_c_consumer_reproduces_golden_steps(tmp_path, golden, solver, variant):
    exe = build(tmp_path)
    pos, ori = golden["positions"], golden["orientations"]
    n = len(pos)
    fibers = tmp_path / "XcT_ref100.in"
    with open(fibers, "w") as fh:
        fh.write("%d\n" % n)
        for p, o in zip(pos, ori):
            fh.write("%.16f %.16f %.16f\n%.16f %.16f %.16f\n" % (*p, *o))
    r = subprocess.run([exe, str(fibers), "2", solver], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.loadtxt(r.stdout.splitlines())
    assert out.shape == (2 * n, 3)
    for got, key in ((out[:n], "POS"), (out[n:], "ORIENT")):
        ref = golden["%s/1_%s" % (variant, key)].reshape(-1)
        err = np.abs(got.reshape(-1) - ref).max() / np.abs(ref).max()
        assert err <= 1e-5, (key, err)
