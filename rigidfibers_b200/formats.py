"""File formats of the reference: the .ini run configuration and the XcT
fibers file, plus the state / velocity / validate-dump writers.

  .ini   sections RUN, SIMULATION, GMRES, BICGSTAB (tests/config.ini:18-37,
         read by runner/cuda_runner.py:18-47)
  XcT    line 1: N; then per fiber one line "x y z" (position) and one line
         "tx ty tz" (orientation) (src/parameters.cc:75-116; the Fortran
         reader fortran/fibers.f95:162-168 also accepts both on one line)
  XcT_res_%05d.out / TcR_res_%05d.out   N, then per fiber two lines with
         8 decimals (src/simulation.cu:530-604)
  validate dumps: one value per line, F16.8 (fortran/fibers.f95:205-303)
"""
import configparser

import numpy as np


class ConfigError(ValueError):
    pass


def read_config(path):
    """Parse a reference .ini into a dict with the reference's key names."""
    cp = configparser.ConfigParser()
    with open(path) as fh:
        cp.read_file(fh)
    try:
        p = {
            "NUMBER_OF_TIMESTEPS": cp.getint("RUN", "NUMBER_OF_TIMESTEPS"),
            "STATE_SAVE_INTERVAL": cp.getint("RUN", "STATE_SAVE_INTERVAL", fallback=0),
            "VELOCITY_SAVE_INTERVAL": cp.getint("RUN", "VELOCITY_SAVE_INTERVAL", fallback=0),
            "TIMESTEP": cp.getfloat("SIMULATION", "TIMESTEP"),
            "SLENDERNESS": cp.getfloat("SIMULATION", "SLENDERNESS"),
            "NUMBER_OF_TERMS_IN_FORCE_EXPANSION": cp.getint("SIMULATION", "NUMBER_OF_TERMS_IN_FORCE_EXPANSION"),
            "NUMBER_OF_QUADRATURE_INTERVALS": cp.getint("SIMULATION", "NUMBER_OF_QUADRATURE_INTERVALS"),
            "NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL": cp.getint("SIMULATION",
                                                                  "NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL"),
            "GMRES_RESTART": cp.getint("GMRES", "RESTART", fallback=10),
            "GMRES_MAX_ITERATIONS": cp.getint("GMRES", "MAX_ITERATIONS", fallback=1000),
            "GMRES_TOLERANCE": cp.getfloat("GMRES", "TOLERANCE", fallback=1e-5),
            "BICGSTAB_MAX_ITERATIONS": cp.getint("BICGSTAB", "MAX_ITERATIONS", fallback=1000),
            "BICGSTAB_TOLERANCE": cp.getfloat("BICGSTAB", "TOLERANCE", fallback=1e-5),
        }
    except (configparser.Error, ValueError) as e:
        raise ConfigError("%s: %s" % (path, e))
    if p["NUMBER_OF_QUADRATURE_POINTS_PER_INTERVAL"] != 3:
        raise ConfigError("%s: only 3 Gauss points per interval are defined" % path)
    if not 1 <= p["NUMBER_OF_TERMS_IN_FORCE_EXPANSION"] <= 8:
        raise ConfigError("%s: NUMBER_OF_TERMS_IN_FORCE_EXPANSION must be in [1, 8]" % path)
    if p["TIMESTEP"] <= 0 or p["SLENDERNESS"] <= 0:
        raise ConfigError("%s: TIMESTEP and SLENDERNESS must be positive" % path)
    return p


def read_fibers(path):
    """Read an XcT file.  Returns (positions (N,3), orientations (N,3)) as float64."""
    with open(path) as fh:
        tokens = fh.read().split()
    if not tokens:
        raise ConfigError("%s: empty fibers file" % path)
    try:
        n = int(tokens[0])
        vals = np.array([float(t) for t in tokens[1:1 + 6 * n]], dtype=np.float64)
    except ValueError as e:
        raise ConfigError("%s: %s" % (path, e))
    if n < 1 or vals.size != 6 * n:
        raise ConfigError("%s: expected %d fibers (%d numbers), found %d numbers" % (path, n, 6 * n, vals.size))
    v = vals.reshape(n, 2, 3)
    return v[:, 0, :].copy(), v[:, 1, :].copy()


def write_fibers(path, pos, ori, fmt="%.8f"):
    """XcT_res style: N, then position and orientation lines per fiber."""
    pos = np.asarray(pos).reshape(-1, 3)
    ori = np.asarray(ori).reshape(-1, 3)
    with open(path, "w") as fh:
        fh.write("%d\n" % pos.shape[0])
        for p, o in zip(pos, ori):
            fh.write(" ".join(fmt % v for v in p) + "\n")
            fh.write(" ".join(fmt % v for v in o) + "\n")


def write_column(path, values):
    """Validate dump: one value per line, Fortran F16.8."""
    with open(path, "w") as fh:
        for v in np.asarray(values, dtype=np.float64).reshape(-1):
            fh.write("%16.8f\n" % v)


def read_column(path):
    return np.loadtxt(path, dtype=np.float64).reshape(-1)
