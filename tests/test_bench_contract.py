"""The bench's reference arm on the CPU: one JSON line with the contract's keys
(the GPU arm needs a B200 and is exercised by the driver)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config0", "--steps", "1",
                        "--warmup", "0", "--ref-rows", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return  # the reference build is absent here
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("config0")


def test_roofline_figures_come_from_the_committed_profiles():
    """The GPU arm's `roofline.traffic` and `roofline.issue` are read from the
    committed ncu summaries: every lifetime-kernel summary carries the
    machine-readable lines, and the traffic scales with the orbits per launch."""
    sys.path.insert(0, str(ROOT))
    import bench
    for name in ("split", "fp64"):
        issue = bench.profiled_issue(name)
        assert issue is not None, name
        assert 0.0 < issue["issue_active_frac"] <= 1.0 and 0.0 < issue["threads_per_instruction"] <= 32.0
        assert abs(issue["lane_frac"] - issue["threads_per_instruction"] / 32.0) < 1e-12
        t1 = bench.profiled_traffic(name)
        # most of the 8-byte lifetime write of a 257^2 x 516 pass (part of it can
        # still sit in the 126 MB L2 when the kernel ends)
        assert t1 and t1 > 0.5 * 8 * 34_081_284
    full = bench.profiled_traffic("split", 34_081_284)
    half = bench.profiled_traffic("split", 34_081_284 // 2)
    assert abs(full - 2 * half) / full < 1e-6


def test_reference_arm_default_is_the_config2_slice():
    """The driver's reference arm (no --workload) times the reference's CPU code on
    the same workload as the GPU arm's default: the config-2 sweep slice."""
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--ref-rows", "1"], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return
    assert d["config"]["workload"] == "config2-slice0-3x32x3"
    assert d["value"] > 0 and d["sigma_points_per_sec"] > 0
    assert d["e2e"]["value"] == d["value"]


def test_integrate_traffic_comes_from_the_committed_profiles():
    """The bench's stages-(b)+(c) roofline reads its DRAM traffic from the committed ncu
    summaries of integrate_flat_kernel: about the 8 algorithmic bytes per orbit."""
    sys.path.insert(0, str(ROOT))
    import bench
    for name in ("split", "fp64"):
        n = 135_797_636  # a 513^2 x 516 pass
        t = bench.profiled_traffic(f"integrate_flat_{name}_config1.md", n)
        assert t is not None and 8 * n <= t <= 1.05 * 8 * n, (name, t)
