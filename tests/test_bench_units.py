"""The algorithmic units bench.py divides by (no GPU needed): the contraction
flops F and compulsory HBM bytes Q of one analysis+synthesis pair,
F = 4 sum_j sum_{l in (bl_lo, bl)} (l+1)^2 (#{n: |n| <= min(N-1,l), N+n odd}
    + #{n: 0 <= n <= min(N-1,l), N+n odd}),
Q = 2*8*(wavelet samples) + 2*16*B(B+1)/2,
at the four workload sizes (alpha = 2, J = Jmax), and the whole-pair roofline
t_min = max(F / P_FP64, Q / BW_HBM)."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from s2dw_b200 import core  # noqa: E402


@pytest.mark.parametrize("B,N,F_gflop,Q_mb", [(64, 3, 0.003548, 1.9), (256, 5, 0.3593, 49.9),
                                              (1024, 4, 17.20, 642.7), (2048, 8, 275.0, 5076.4)])
def test_pair_units(B, N, F_gflop, Q_mb):
    J = core.s2dw_core_comp_Jmax(B, 2.0)
    r = bench.pair_roofline(B, N, 2.0, J, t_ms=1.0, fp64_peak_tflops=35.0)
    assert abs(r["flops"] / 1e9 - F_gflop) <= 1e-3 * F_gflop
    assert abs(r["bytes"] / 1e6 - Q_mb) <= 0.05 + 1e-4 * Q_mb
    assert r["t_min_ms"] == max(r["t_flops_ms"], r["t_hbm_ms"])
    assert r["frac"] == r["t_min_ms"] / 1.0


def test_contraction_flops_split_by_kind():
    # analysis counts +-n, synthesis n >= 0: for N = 4 (n = 1, 3 used) the
    # analysis does twice the synthesis MACs once l >= 3
    ana, syn = bench.contraction_flops_per_scale(1024, 4, 2.0, 10)
    assert len(ana) == len(syn) == 11
    assert abs(sum(ana) / sum(syn) - 2.0) < 1e-3


def test_reference_arm_loads_only_the_oracle():
    """`bench.py --impl reference` times full, unsampled CPU pairs of the
    restatement and never loads the CUDA library (small B here)."""
    import json
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--B', '64', '--N', '3', "
            "'--steps', '2', '--warmup', '1']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'cuda_lib': 'libs2dw_cuda' in maps, 'oracle_lib': 'libs2dw_oracle' in maps}))")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    line, libs = lines[0], lines[-1]
    assert libs == {"cuda_lib": False, "oracle_lib": True}
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["config"]["recon_err"] < 1e-10
    assert "unsampled" in line["cpu_baseline"]["sample"]
    assert abs(line["ms_per_step"] * line["value"] - 1e3) < 1e-6 * 1e3
