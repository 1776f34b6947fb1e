"""bench.py's per-stage roofline arithmetic (host only)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_assembly_flop_count():
    # Q^2 (25 + 12 M + 18) + 12 M^2 Q + 6 M Q + 25 * 27 at M = 5, Q = 24
    assert bench.asm_flops_per_ordered_pair() == 576 * 103 + 7200 + 720 + 675 == 67923
    assert bench.asm_flops_per_ordered_pair(M=3, Q=24) == 576 * (25 + 36 + 18) + 12 * 9 * 24 + 6 * 3 * 24 + 675


def test_kernel_rooflines_of_a_mixed_step():
    N, hbm = 4000, 6434.2
    head = {"stage": {"assemble_system": 112.0, "solve_system": 125.0, "update_velocities": 7.7,
                      "update_fibers": 0.1},
            "iters": 217, "refinements": 20, "ms": 245.0, "steps": 10}
    k = bench.kernel_rooflines(N, head, hbm, True, {"fibers": 2000, "direct": {"tflops": 28.0}})
    pairs = N * (N - 1) / 2
    # executed flops per unordered pair from the kernel's instruction mix
    # (thread instructions FFMA 7.15 G, FMUL 1.69 G, FADD 1.92 G for 499,500 pairs)
    per_pair = (7.15e9 * 2 + 1.69e9 + 1.92e9) / 499500
    assert 35000 < per_pair < 37000
    assert abs(bench.ASM_EXEC_FLOPS_PER_PAIR - per_pair) < 1e-9
    flops = per_pair * pairs
    assert abs(k["assembly"]["achieved_tflops"] - flops / 11.2e-3 / 1e12) < 1e-6
    assert abs(k["assembly"]["frac"] - flops / 11.2e-3 / 1e12 / bench.NOMINAL_FP32_TFLOPS) < 1e-9
    assert k["assembly"]["frac"] < 1.0
    assert abs(k["assembly"]["store_gbs"] - pairs * 1168 / 11.2e-3 / 1e9) < 1e-6
    assert abs(k["velocities"]["achieved_gbs"] - pairs * 480 / 0.77e-3 / 1e9) < 1e-6
    bound = 1e3 * (flops / (bench.NOMINAL_FP32_TFLOPS * 1e12) + (21.7 * pairs * 300 + 2 * pairs * 600) / (hbm * 1e9)
                   + pairs * 480 / (hbm * 1e9))
    assert abs(k["step"]["bound_ms"] - bound) < 1e-9
    assert abs(k["step"]["frac"] - bound / 24.5) < 1e-9
    assert abs(k["lu"]["frac"] - 28.0 / bench.NOMINAL_TF32_TFLOPS) < 1e-12


def test_kernel_rooflines_of_a_dense_step():
    head = {"stage": {"assemble_system": 14.0, "solve_system": 49.0, "update_velocities": 10.0,
                      "update_fibers": 0.0},
            "iters": 21, "refinements": 0, "ms": 73.0, "steps": 1}
    k = bench.kernel_rooflines(4000, head, 6434.2, False)
    assert "velocities" not in k and "lu" not in k
    assert abs(k["assembly"]["store_gbs"] - 4.0 * 60000 ** 2 / 14e-3 / 1e9) < 1e-6
