"""bench.py's helpers (CPU): the reader of the committed ncu summaries (the
DRAM traffic per tet of its roofline entry, every kernel of a pass added;
a missing summary reported rather than guessed; the executed FP64 flops per
tet of the compute figure), the algorithmic bytes of
the scope table, the reference arm's slabs (every cell layer of the
workload exactly once) and its JSON line."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_dram_traffic_per_tet_from_profile():
    # assemble_rows_kernel_quench48.md: one kernel, 397.439488 MB read and
    # 146.457856 MB written on the 663,552-tet case
    per_tet, src = bench.ncu_dram_per_tet("assemble_rows_kernel_quench48.md", 663552)
    assert per_tet is not None and "profiles/assemble_rows_kernel_quench48.md" in src
    assert abs(per_tet * 663552 - (397.439488e6 + 146.457856e6)) < 1.0


def test_dram_traffic_adds_every_kernel_of_a_summary(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "two.md").write_text("| `dram__bytes_read.sum` | 1.5 Mbyte |\n| `dram__bytes_write.sum` | 500 Kbyte |\n"
                                 "| `dram__bytes_read.sum` | 2 Gbyte |\n| `dram__bytes_write.sum` | 10 byte |\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    per_tet, _ = bench.ncu_dram_per_tet("two.md", 10)
    assert abs(per_tet * 10 - (1.5e6 + 5e5 + 2e9 + 10)) < 1e-3


def test_missing_summaries_are_reported():
    per_tet, why = bench.ncu_dram_per_tet("no_such_summary.md", 1)
    assert per_tet is None and "no ncu summary" in why
    fl, why = bench.ncu_flops_per_tet("no_such_summary.md")
    assert fl is None and "no ncu summary" in why


def test_fp64_flops_per_tet_add_every_kernel(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "f.md").write_text("| element pass | 1 | 2 | 3 | 4 | `fp64_flops_per_tet` 4612 |\n"
                               "| row pass | 1 | 2 | 3 | 4 | `fp64_flops_per_tet` 1839 |\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    fl, src = bench.ncu_flops_per_tet("f.md")
    assert fl == 4612 + 1839 and "profiles/f.md" in src
    (prof / "g.md").write_text("no counts here\n")
    fl, why = bench.ncu_flops_per_tet("g.md")
    assert fl is None and "no FP64 flop counts" in why


def test_algorithmic_bytes_of_the_scope_table():
    """The pass and SpMV bytes at config 3 (128^3 x6 tets): NS+VOF assembly
    6.80 GB in FP64 and 3.51 GB in FP32; preconditioned SpMV 3.37 GB FP32."""
    E, N, nnz = 12582912, 2146689, 31802497
    assert abs(bench.assembly_pass_bytes(E, N, nnz, 8) / 1e9 - 6.80) < 0.005
    assert abs(bench.assembly_pass_bytes(E, N, nnz, 4) / 1e9 - 3.507) < 0.001
    assert abs(bench.spmv_bytes(N, nnz, 4) / 1e9 - 3.37) < 0.01


def test_reference_slabs_cover_the_workload():
    for n, parts in ((128, 16), (128, 12), (16, 32), (7, 3), (1, 1)):
        sl = bench.slab_layers(n, parts)
        assert sum(nl for _, nl in sl) == n and sl[0][0] == 0
        assert all(k0 + nl == sl[i + 1][0] for i, (k0, nl) in enumerate(sl[:-1]))
        assert max(nl for _, nl in sl) - min(nl for _, nl in sl) <= 1 and min(nl for _, nl in sl) >= 1


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


class _RecordingContext:
    """Stands in for api.Context in the streamed end-to-end loop: records
    the calls in order."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return lambda *a, **k: self.calls.append(name)


def _count(calls, name):
    return sum(c == name for c in calls)


def test_streamed_steps_hold_every_steps_copies():
    """bench.streamed_steps: K steps hold K uploads of the fields, K passes
    and K read-backs of both residuals, primed (the steady state of a time
    loop) or not; every step commits its fields before its pass, stages
    the next step's only after that commit, and the loop ends with the
    copies synchronized."""
    from oversetdevfort_b200 import _ffi as F
    for primed in (False, True):
        for K in (1, 3, 5):
            ctx = _RecordingContext()
            bench.streamed_steps(ctx, F, {"ug": None}, None, None, K, primed)
            c = ctx.calls
            assert _count(c, "stage_fields") == K
            assert _count(c, "commit_staged") == K
            assert _count(c, "assemble_async") == K and _count(c, "assemble_wait") == K
            assert _count(c, "get_rhs_async") == 2 * K
            assert c[-1] == "sync_copies" and _count(c, "sync_copies") == 1
            commits = [i for i, n in enumerate(c) if n == "commit_staged"]
            passes = [i for i, n in enumerate(c) if n == "assemble_async"]
            assert all(cm < ps for cm, ps in zip(commits, passes))
            stages = [i for i, n in enumerate(c) if n == "stage_fields"]
            inside = [s for s in stages if s > commits[0]]
            # primed: each step stages after its own commit; unprimed: the
            # first upload comes before the loop, the last step stages nothing
            assert len(inside) == (K if primed else K - 1)
