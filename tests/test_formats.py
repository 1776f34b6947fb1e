"""The reference's file formats: .ini and XcT (tests/config.ini,
tests/XcT_*.in; src/parameters.cc:75-116)."""
import numpy as np
import pytest

from rigidfibers_b200 import formats as F

INI = """[RUN]
NUMBER_OF_TIMESTEPS=10
STATE_SAVE_INTERVAL=1
VELOCITY_SAVE_INTERVAL=1

[SIMULATION]
TIMESTEP=0.1
SLENDERNESS=0.01
NUMBER_OF_TERMS_IN_FORCE_EXPANSION=5
NUMBER_OF_QUADRATURE_INTERVALS=8
NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL=3

[GMRES]
RESTART=10
MAX_ITERATIONS=1000
TOLERANCE=1e-5

[BICGSTAB]
MAX_ITERATIONS=1000
TOLERANCE=1e-5
"""


def test_read_config(tmp_path):
    p = tmp_path / "c.ini"
    p.write_text(INI)
    c = F.read_config(str(p))
    assert c["NUMBER_OF_TIMESTEPS"] == 10 and c["TIMESTEP"] == 0.1 and c["GMRES_TOLERANCE"] == 1e-5


def test_missing_save_interval_defaults(tmp_path):
    # tests/config400.ini etc. in the reference lack STATE_SAVE_INTERVAL
    p = tmp_path / "c.ini"
    p.write_text(INI.replace("STATE_SAVE_INTERVAL=1\n", ""))
    assert F.read_config(str(p))["STATE_SAVE_INTERVAL"] == 0


@pytest.mark.parametrize("bad", ["NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL=3", "TIMESTEP=0.1",
                                 "NUMBER_OF_TERMS_IN_FORCE_EXPANSION=5"])
def test_bad_config(tmp_path, bad):
    repl = {"NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL=3": "NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL=4",
            "TIMESTEP=0.1": "TIMESTEP=abc",
            "NUMBER_OF_TERMS_IN_FORCE_EXPANSION=5": "NUMBER_OF_TERMS_IN_FORCE_EXPANSION=9"}[bad]
    p = tmp_path / "c.ini"
    p.write_text(INI.replace(bad, repl))
    with pytest.raises(F.ConfigError):
        F.read_config(str(p))


def test_xct_roundtrip(tmp_path, golden):
    pos, ori = golden["positions"], golden["orientations"]
    p = tmp_path / "x.in"
    F.write_fibers(str(p), pos, ori, fmt="%.16f")
    pos2, ori2 = F.read_fibers(str(p))
    assert np.array_equal(pos, pos2) and np.array_equal(ori, ori2)


def test_xct_both_layouts(tmp_path):
    # two lines per fiber (src/parameters.cc) or six numbers on one line (Fortran list-directed read)
    a = tmp_path / "a.in"
    a.write_text("2\n0 0 0\n0 0 1\n1 2 3\n1 0 0\n")
    b = tmp_path / "b.in"
    b.write_text("2\n0 0 0 0 0 1\n1 2 3 1 0 0\n")
    pa, oa = F.read_fibers(str(a))
    pb, ob = F.read_fibers(str(b))
    assert np.array_equal(pa, pb) and np.array_equal(oa, ob) and pa[1, 2] == 3


@pytest.mark.parametrize("text", ["", "3\n0 0 0\n0 0 1\n", "x\n"])
def test_xct_malformed(tmp_path, text):
    p = tmp_path / "m.in"
    p.write_text(text)
    with pytest.raises(F.ConfigError):
        F.read_fibers(str(p))


def test_column_dump(tmp_path):
    p = tmp_path / "v.out"
    F.write_column(str(p), [1.0, -0.123456789])
    assert open(str(p)).read() == "      1.00000000\n     -0.12345679\n"
    assert np.allclose(F.read_column(str(p)), [1.0, -0.12345679])
