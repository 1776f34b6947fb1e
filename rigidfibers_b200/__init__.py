"""B200-native rigid-fiber time step (Tornberg-Gustavsson slender-body
method): CUDA kernels for sm_100a behind a C ABI (include/rigidfibers.h).

    from rigidfibers_b200 import Simulation, Config
"""
from .formats import read_config, read_fibers, write_fibers  # noqa: F401


def __getattr__(name):
    # the CUDA library is loaded on first use of the simulation API
    if name in ("Simulation", "Config"):
        from . import simulation
        return getattr(simulation, name)
    if name == "RigidFibersError":
        from ._capi import RigidFibersError
        return RigidFibersError
    raise AttributeError(name)
