"""CPU-side checks of the C ABI library: it loads, exports every entry point
that include/rigidfibers.h declares, and its host-side logic (defaults,
argument validation, status strings) works without a GPU."""
import ctypes
import os
import re

import pytest

from rigidfibers_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rigidfibers.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_step_seam():
    names = declared_functions()
    for n in ["rf_create", "rf_destroy", "rf_assemble", "rf_solve", "rf_update_velocities", "rf_update_fibers",
              "rf_step", "rf_get_state", "rf_get_velocities", "rf_get_system", "rf_get_solution", "rf_last_stats"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = C.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in C.SIGNATURES, "binding lacks " + name


def test_defaults_match_reference_config():
    lib = C.load()
    c = C.rf_config()
    assert lib.rf_config_default(ctypes.byref(c)) == 0
    assert c.timestep == 0.1 and c.slenderness == 0.01
    assert c.number_of_terms_in_force_expansion == 5 and c.number_of_quadrature_intervals == 8
    assert c.gmres_restart == 10 and c.gmres_max_iterations == 1000 and c.gmres_tolerance == 1e-5


def test_status_strings():
    lib = C.load()
    assert lib.rf_status_string(0) == b"ok"
    assert lib.rf_status_string(C.RF_E_NOCONV) == b"solver did not converge"


@pytest.mark.parametrize("field,value", [("number_of_terms_in_force_expansion", 9),
                                         ("number_of_quadrature_points_per_interval", 4),
                                         ("slenderness", -1.0), ("gmres_restart", 0)])
def test_create_rejects_bad_config_before_touching_the_device(field, value):
    import numpy as np
    lib = C.load()
    c = C.rf_config()
    lib.rf_config_default(ctypes.byref(c))
    setattr(c, field, value)
    pos = np.zeros(3)
    h = ctypes.c_void_p()
    rc = lib.rf_create(ctypes.byref(c), 1, C.ptr(pos), C.ptr(pos), ctypes.byref(h))
    assert rc in (C.RF_E_INPUT, C.RF_E_UNSUPPORTED)
    assert not h.value
    assert lib.rf_last_error()


def test_null_handle_is_an_input_error():
    lib = C.load()
    assert lib.rf_assemble(None) == C.RF_E_INPUT
    assert lib.rf_destroy(None) == C.RF_E_INPUT


@pytest.mark.parametrize("sms", [148, 1000, 4096])
@pytest.mark.parametrize("R", [1, 64, 1500, 4099, 30000, 60000, 131072])
def test_noalloc_plan_fits_its_scratch_and_covers_every_column(R, sms):
    """The allocation-free matvec caps its column splits so that splits x R
    partial rows fit the fixed 8 MiB (2^21 float) scratch array; on a GPU with
    many more SMs than a B200 the uncapped plan would overflow it.  The capped
    plan must still cover every column exactly once."""
    lib = C.load()
    splits, cps = ctypes.c_int(), ctypes.c_int64()
    assert lib.rf_debug_noalloc_plan(R, sms, ctypes.byref(splits), ctypes.byref(cps)) == C.RF_OK
    s, c = splits.value, cps.value
    assert s >= 1 and c >= 1
    assert s * R <= 2 * 1024 * 1024
    # split k covers [k*c, min(R, (k+1)*c)): all R columns, none empty
    assert (s - 1) * c < R <= s * c


def test_noalloc_plan_caps_splits_on_large_gpus():
    lib = C.load()
    splits, cps = ctypes.c_int(), ctypes.c_int64()
    lib.rf_debug_noalloc_plan(60000, 148, ctypes.byref(splits), ctypes.byref(cps))
    b200 = splits.value
    lib.rf_debug_noalloc_plan(60000, 4096, ctypes.byref(splits), ctypes.byref(cps))
    assert splits.value * 60000 <= 2 * 1024 * 1024 and splits.value >= b200


def test_noalloc_plan_rejects_sizes_beyond_its_scratch():
    lib = C.load()
    splits, cps = ctypes.c_int(), ctypes.c_int64()
    assert lib.rf_debug_noalloc_plan(131073, 148, ctypes.byref(splits), ctypes.byref(cps)) == C.RF_E_INPUT
    assert lib.rf_debug_noalloc_plan(0, 148, ctypes.byref(splits), ctypes.byref(cps)) == C.RF_E_INPUT


@pytest.mark.parametrize("field,value", [("integration", 1), ("solver", 2), ("precision", 6)])
def test_matrix_free_mode_rejects_what_it_does_not_support(field, value):
    """The matrix-free mode recomputes the symmetric pair blocks of numerical
    integration inside GMRES or BiCGSTAB: analytical integration and the
    direct solver (which factors a stored matrix) are refused before the
    device is touched, as is an unknown precision."""
    import numpy as np
    lib = C.load()
    c = C.rf_config()
    lib.rf_config_default(ctypes.byref(c))
    c.precision = C.PRECISIONS["matrix_free"]
    setattr(c, field, value)
    pos = np.zeros(3)
    h = ctypes.c_void_p()
    rc = lib.rf_create(ctypes.byref(c), 1, C.ptr(pos), C.ptr(pos), ctypes.byref(h))
    assert rc in (C.RF_E_INPUT, C.RF_E_UNSUPPORTED)
    assert not h.value


def test_recompute_modes_store_the_16_bit_copy_only():
    """RF_PREC_MIXED_*_RECOMPUTE keep the 16-bit pair records (304 bytes per
    unordered pair) and drop the FP32 blocks (864 bytes per pair) and the
    structured velocity partials; they take what the mixed modes take (GMRES or
    BiCGSTAB, numerical integration) and refuse the rest before the device is
    touched."""
    import numpy as np
    lib = C.load()

    def est(prec, n):
        c = C.rf_config()
        lib.rf_config_default(ctypes.byref(c))
        c.precision = C.PRECISIONS[prec]
        return lib.rf_device_bytes_estimate(ctypes.byref(c), n)

    n = 2000
    pairs = n * (n - 1) // 2
    for p16 in ("fp16", "bf16"):
        lean, full = est("mixed_%s_recompute" % p16, n), est("mixed_" + p16, n)
        assert lean >= pairs * 304
        assert full - lean >= pairs * 864 * 0.99
        assert lean < 0.3 * full
    for field, value in (("integration", 1), ("solver", 2), ("number_of_quadrature_intervals", 4)):
        c = C.rf_config()
        lib.rf_config_default(ctypes.byref(c))
        c.precision = C.PRECISIONS["mixed_fp16_recompute"]
        setattr(c, field, value)
        pos = np.zeros(3)
        h = ctypes.c_void_p()
        rc = lib.rf_create(ctypes.byref(c), 1, C.ptr(pos), C.ptr(pos), ctypes.byref(h))
        assert rc in (C.RF_E_INPUT, C.RF_E_UNSUPPORTED)
        assert not h.value


def test_matrix_free_footprint_grows_with_the_vectors_only():
    """Without a stored operator the device footprint is O(N) vectors plus
    O(N^2 / 8) partial rows: at N=16000 well under the 155 GB the structured
    operator would take, and far under the dense FP32 matrix."""
    lib = C.load()
    c = C.rf_config()
    lib.rf_config_default(ctypes.byref(c))
    sizes = {}
    for prec in ("fp32", "mixed_fp16", "matrix_free"):
        c.precision = C.PRECISIONS[prec]
        sizes[prec] = [lib.rf_device_bytes_estimate(ctypes.byref(c), n) for n in (4000, 16000)]
    assert sizes["matrix_free"][0] < sizes["mixed_fp16"][0] / 10 < sizes["fp32"][0]
    assert sizes["matrix_free"][1] < 8e9 < 1.5e11 < sizes["mixed_fp16"][1]
