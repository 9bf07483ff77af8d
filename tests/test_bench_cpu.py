"""Host logic of bench.py, on the CPU: the per-kernel roofline grouping, the committed
DRAM/algorithmic traffic ratio, the measured peaks, and the command-line flags."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_kernel_rooflines_groups_and_rates():
    # (name, device ms, algorithmic bytes) per profiled launch
    entries = [("schur_operator", 2.0, 4e9), ("schur_operator", 2.0, 4e9), ("schur_operator", 0.1, 1e8),
               ("bicgstab_update", 1.0, 5e9), ("graph_sweep", 0.5, 1e9)]
    out = {(k["kernel"], k["scope"]): k for k in bench.kernel_rooflines(entries)}
    op = out[("schur_operator", "all")]
    assert op["launches"] == 3 and op["ms"] == pytest.approx(4.1)
    assert op["achieved"] == pytest.approx((8e9 + 1e8) / 4.1e-3 / 1e9)
    big = out[("schur_operator", "largest_level_group")]
    # records of at least half the class's largest per-launch bytes
    assert big["launches"] == 2 and big["bytes_per_launch"] == pytest.approx(4e9)
    assert big["achieved"] == pytest.approx(2000.0)
    assert out[("bicgstab_update", "largest_level_group")]["launches"] == 1
    assert ("graph_sweep", "largest_level_group") not in out
    assert out[("graph_sweep", "all")]["achieved"] == pytest.approx(2000.0)


def test_traffic_ratio_matches_its_capture():
    tpb = bench.traffic_per_byte()
    path = os.path.join(REPO, "profiles", "schur_operator_largest_group_n20_x64_traffic.json")
    with open(path) as f:
        rec = json.load(f)
    assert tpb == rec["dram_bytes_per_algorithmic_byte"]
    assert tpb == pytest.approx(rec["dram_bytes"] / rec["algorithmic_bytes"], rel=1e-3)
    # DRAM bytes must not fall below the algorithmic count of a full-size launch
    assert tpb >= 1.0


def test_peaks_are_positive():
    hbm, kind = bench.peaks()
    assert hbm > 1000.0 and kind in ("measured", "fallback")
    assert bench.bf16_peak() > 100.0


def test_command_line_flags():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--help"], capture_output=True,
                         text=True, timeout=120, check=True).stdout
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--method", "--no-compare", "--no-cpu-baseline",
                 "--no-many", "--batch", "--profile-run", "--profile-table", "--profile-mlp"):
        assert flag in out, flag
