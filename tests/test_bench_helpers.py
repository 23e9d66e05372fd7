"""The bench's readers of the committed ncu summaries (CPU): the DRAM
traffic and the executed FP32 flops per tet that bench.py puts into its
roofline entries come out of profiles/ with the expected values, and a
missing summary is reported rather than guessed."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_dram_traffic_per_tet_from_profile():
    per_tet, src = bench.ncu_traffic_per_tet("assemble_rows_kernel_quench128_dram.md", 12582912)
    assert per_tet is not None and "profiles/assemble_rows_kernel_quench128_dram.md" in src
    # 8.28 GB per launch of the 128^3 case
    assert abs(per_tet * 12582912 / 1e9 - 8.28) < 0.01


def test_fp32_flops_per_tet_from_profile():
    per_tet, src = bench.ncu_flops_per_tet("assemble_rows_kernel_quench48_flops.md", 663552)
    assert per_tet == 4948.0 and "FFMA" in src


def test_missing_summaries_are_reported():
    assert bench.ncu_traffic_per_tet("no_such_summary.md", 1) == (None, "no ncu summary")
    assert bench.ncu_flops_per_tet("no_such_summary.md", 1) == (None, "no ncu summary")


def test_reference_arm_counts_usable_cores():
    import os
    import bench
    n = bench._host_cores()
    assert 1 <= n <= (os.cpu_count() or n)
    if hasattr(os, "sched_getaffinity"):
        assert n == len(os.sched_getaffinity(0))


def test_reference_arm_json_line():
    """bench.py --impl reference (CPU, a small cube): one JSON line with the
    contract's keys, impl "reference", a cpu_baseline of kind "port" and an
    e2e with no host-device traffic."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    res = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "3",
                          "--n", "16"], capture_output=True, text=True, timeout=600, cwd=root)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_own_arm_fails_without_a_device():
    """bench.py's own arm has no CPU path: without a CUDA device it exits
    non-zero on ovs_create's OVS_ERR_NODEVICE and prints no bench line."""
    import subprocess
    import sys
    from pathlib import Path
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    root = Path(__file__).resolve().parent.parent
    res = subprocess.run([sys.executable, str(root / "bench.py"), "--steps", "1", "--warmup", "3", "--n", "8",
                          "--no-solve", "--no-adjoint", "--no-hex", "--no-cpu"], capture_output=True, text=True,
                         timeout=600, cwd=root)
    assert res.returncode != 0
    assert "no CUDA device" in res.stderr
    assert not [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
