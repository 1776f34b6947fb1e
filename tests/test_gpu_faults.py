"""Failure detection without a GPU fault: device-side waits are bounded and
report RF_E_TIMEOUT (forced here by a zero wait limit, so the waits give up
before the copies / tensor-core products they wait for complete), allocation
failures report RF_E_OOM, and in both cases the library stays usable."""
import numpy as np
import pytest

from rigidfibers_b200.generate import sphere_layout

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    yield lib
    lib.rf_debug_set_device_wait_limit(-1)
    lib.rf_debug_fail_allocation_after(-1)


def _sim(**kw):
    from rigidfibers_b200 import Config, Simulation
    pos, ori = sphere_layout(200, 5.0, seed=41)
    return Simulation(Config(**kw), pos, ori)


@pytest.mark.parametrize("kw", [dict(precision="mixed_fp16"), dict(solver="direct", integration="analytical")])
def test_bounded_wait_reports_timeout_and_recovers(lib, kw):
    from rigidfibers_b200 import _capi as C
    sim = _sim(**kw)
    sim.step(0)                                   # normal step first
    lib.rf_debug_set_device_wait_limit(0)
    with pytest.raises(C.RigidFibersError) as e:
        sim.step(1)
    assert e.value.status == C.RF_E_TIMEOUT
    lib.rf_debug_set_device_wait_limit(-1)
    sim.step(1)                                   # the handle and the context still work
    p, o = sim.state()
    assert np.isfinite(p).all() and np.isfinite(o).all()


def test_injected_allocation_failure(lib):
    from rigidfibers_b200 import _capi as C
    for n in (0, 3, 11):
        lib.rf_debug_fail_allocation_after(n)
        with pytest.raises(C.RigidFibersError) as e:
            _sim(precision="mixed_bf16")
        assert e.value.status == C.RF_E_OOM
    lib.rf_debug_fail_allocation_after(-1)
    sim = _sim(precision="mixed_bf16")
    sim.step(0)
