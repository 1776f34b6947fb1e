"""Host-side logic of the serving loop (rf_server_*) without a GPU: the
admission estimate, refusal of requests that cannot fit or are invalid, the
request state machine and percentile bookkeeping."""
import ctypes

import numpy as np
import pytest

from rigidfibers_b200 import _capi as C


def _cfg(**kw):
    from rigidfibers_b200 import Config
    return Config(**kw)


def test_device_bytes_estimate_scales_with_the_system():
    from rigidfibers_b200.server import device_bytes
    fp32 = [device_bytes(_cfg(), n) for n in (100, 200, 400)]
    mixed = [device_bytes(_cfg(precision="mixed_bf16"), n) for n in (100, 200, 400)]
    for n, b in zip((100, 200, 400), fp32):
        R = 15 * n
        assert b >= R * R * 4          # the dense (15N)^2 FP32 matrix
        assert b <= 3 * R * R * 4
    # the dense matrix dominates: x4 per doubling of N, asymptotically
    assert 3.0 < fp32[2] / fp32[1] < 4.2
    # one FP32 + one 16-bit block set per unordered pair: about 2/3 of the dense FP32 matrix
    assert 0.6 < mixed[2] / fp32[2] < 0.75
    direct = device_bytes(_cfg(solver="direct"), 200)
    assert direct > fp32[1] + (15 * 200) ** 2 * 4 * 0.99   # LU factors beside A


def test_estimate_rejects_invalid_configuration():
    lib = C.load()
    c = _cfg(number_of_terms_in_force_expansion=9)
    assert lib.rf_device_bytes_estimate(ctypes.byref(c._c), 10) == -1
    assert lib.rf_device_bytes_estimate(ctypes.byref(_cfg()._c), 0) == -1


def test_server_refuses_what_cannot_run():
    from rigidfibers_b200.server import Server, device_bytes
    pos = np.zeros((20, 3))
    ori = np.tile([0.0, 0.0, 1.0], (20, 1))
    need = device_bytes(_cfg(), 20)
    with Server(max_active=2, hbm_budget_bytes=need - 1) as srv:
        with pytest.raises(C.RigidFibersError) as e:
            srv.submit(_cfg(), pos, ori, 3)
        assert e.value.status == C.RF_E_OOM
        with pytest.raises(C.RigidFibersError) as e:
            srv.submit(_cfg(precision="mixed_fp16", integration="analytical"), pos, ori, 3)
        assert e.value.status == C.RF_E_INPUT
        with pytest.raises(C.RigidFibersError):
            srv.poll(12345)
        st = srv.stats()
        assert st["completed"] == 0 and st["queued"] == 0 and st["steps"] == 0


def test_server_config_validation():
    lib = C.load()
    sc = C.rf_server_config(max_active=0, hbm_budget_bytes=1 << 30)
    s = ctypes.c_void_p()
    assert lib.rf_server_create(ctypes.byref(sc), ctypes.byref(s)) == C.RF_E_INPUT
    sc = C.rf_server_config(max_active=4, hbm_budget_bytes=0)
    assert lib.rf_server_create(ctypes.byref(sc), ctypes.byref(s)) == C.RF_E_INPUT
    sc = C.rf_server_config(max_active=4, hbm_budget_bytes=1 << 30, reserve_bytes=-1)
    assert lib.rf_server_create(ctypes.byref(sc), ctypes.byref(s)) == C.RF_E_INPUT


def test_server_defaults_reserve_a_quarter_of_the_budget():
    lib = C.load()
    sc = C.rf_server_config()
    assert lib.rf_server_config_default(ctypes.byref(sc)) == C.RF_OK
    assert sc.reserve_bytes == sc.hbm_budget_bytes // 4
    assert sc.use_cuda_graphs == 2 and sc.max_active == 8
    assert lib.rf_server_step_times(None, 1, None, 0, ctypes.byref(ctypes.c_int())) == C.RF_E_INPUT


def test_requests_fail_cleanly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present; the GPU tests cover execution")
    from rigidfibers_b200.server import Server
    pos = np.random.default_rng(0).uniform(-3, 3, (10, 3))
    ori = np.tile([0.0, 0.0, 1.0], (10, 1))
    with Server(max_active=2, hbm_budget_bytes=1 << 34) as srv:
        ids = [srv.submit(_cfg(), pos, ori, 2) for _ in range(5)]
        srv.drain(timeout=60)
        assert [srv.poll(i)[0] for i in ids] == ["failed"] * 5
        with pytest.raises(C.RigidFibersError):
            srv.result(ids[0])
        st = srv.stats()
        assert st["failed"] == 5 and st["active"] == 0


def test_pack_config_and_validation():
    lib = C.load()
    sc = C.rf_server_config()
    assert lib.rf_server_config_default(ctypes.byref(sc)) == C.RF_OK
    assert sc.pack_max_fibers == 128 and sc.pack_max_members >= 1
    sc.pack_max_fibers = 64
    sc.pack_max_members = 0
    s = ctypes.c_void_p()
    assert lib.rf_server_create(ctypes.byref(sc), ctypes.byref(s)) == C.RF_E_INPUT
    # packed entry points check their arguments before touching a device
    assert lib.rf_solve_packed(None, 1) == C.RF_E_INPUT
    hs = (ctypes.c_void_p * 1)()
    assert lib.rf_solve_packed(hs, 0) == C.RF_E_INPUT
    assert lib.rf_solve_packed(hs, 1) == C.RF_E_INPUT          # a null handle
    ts = (ctypes.c_int * 1)()
    st = (ctypes.c_int * 1)()
    assert lib.rf_step_packed(hs, ts, 1, st) == C.RF_E_INPUT


def test_packed_requests_fail_cleanly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present; the GPU tests cover execution")
    from rigidfibers_b200.server import Server
    pos = np.random.default_rng(1).uniform(-3, 3, (12, 3))
    ori = np.tile([0.0, 0.0, 1.0], (12, 1))
    with Server(max_active=2, hbm_budget_bytes=1 << 34, pack_max_fibers=64) as srv:
        ids = [srv.submit(_cfg(precision="mixed_bf16"), pos, ori, 2) for _ in range(4)]
        ids.append(srv.submit(_cfg(), pos, ori, 2))                 # FP32: not packed
        srv.drain(timeout=60)
        assert [srv.poll(i)[0] for i in ids] == ["failed"] * 5
        assert srv.stats()["active"] == 0


def test_pack_plan_gives_large_members_clusters():
    """rf_debug_pack_plan: a member's cluster doubles (1, 2, 4, 8 CTAs) while
    the pack fits the multiprocessors and each CTA keeps two storage tiles."""
    lib = C.load()

    def plan(fibers, sms):
        n = len(fibers)
        f = (ctypes.c_int * n)(*fibers)
        c = (ctypes.c_int * n)()
        assert lib.rf_debug_pack_plan(f, n, sms, c) == C.RF_OK
        return list(c)

    assert plan([128], 148) == [8]
    assert plan([64], 148) == [4]          # 10 tiles: 4 CTAs keep two each, 8 would not
    assert plan([48], 148) == [2]
    assert plan([32], 148) == [1]
    assert plan([16] * 100, 148) == [1] * 100
    assert plan([128] * 150, 148) == [1] * 150   # more members than multiprocessors
    assert plan([128, 128], 4) == [2, 2]
    assert plan([256], 148) == [8]
    assert plan([200] * 150, 148) == [2] * 150   # above 128 fibers: never fewer than two CTAs
    rng = np.random.default_rng(3)
    for _ in range(50):
        n = int(rng.integers(1, 200))
        sms = int(rng.integers(1, 300))
        fibers = [int(v) for v in rng.integers(1, 257, n)]
        c = plan(fibers, sms)
        least = [2 if f > 128 else 1 for f in fibers]
        assert sum(c) <= max(sum(least), sms)
        for f, k, k0 in zip(fibers, c, least):
            t = (f + 15) // 16
            assert k in (1, 2, 4, 8) and k >= k0 and (k == k0 or t * (t + 1) // 2 >= 2 * k)
    f = (ctypes.c_int * 2)(16, 257)
    c = (ctypes.c_int * 2)()
    assert lib.rf_debug_pack_plan(f, 2, 148, c) == C.RF_E_INPUT
    assert lib.rf_debug_pack_plan(f, 1, 0, c) == C.RF_E_INPUT
