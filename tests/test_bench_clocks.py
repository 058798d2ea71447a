"""bench.py's clock record (host logic, CPU): nvidia-smi samples are kept only
when they fall inside the timed region of the path asked for, their median SM
clock and the throttle reasons seen there are reported, and all samples are
used when none fell inside. Also the run of the suite's other configurations
(one child process each, failures recorded, a time budget), and the reference
arm's line (the headline's metric and workload on the reference CPU path)."""
import datetime
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

import bench  # noqa: E402


def _line(t, mhz, power_cap):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    cap = "Active" if power_cap else "Not Active"
    return f"{ts}, {mhz}, 1965, 700.0, 0x4, Not Active, Not Active, Not Active, {cap}"


def test_samples_inside_the_path_window(tmp_path, monkeypatch):
    t0 = 1_800_000_000.0
    lines = [_line(t0 + 0.00, 1965, False),   # before the timed regions
             _line(t0 + 1.00, 1965, False),   # DMMA window
             _line(t0 + 1.02, 1965, False),
             _line(t0 + 2.00, 1425, True),    # Ozaki window
             _line(t0 + 2.02, 1500, True),
             _line(t0 + 2.04, 1455, True),
             _line(t0 + 3.00, 1965, False)]   # after
    clk = bench.ClockSampler(0)
    clk.path = tmp_path / "clocks.csv"
    clk.path.write_text("\n".join(lines) + "\n")
    monkeypatch.setattr(bench, "TIMED_WINDOWS", [(1, t0 + 0.9, t0 + 1.1), (2, t0 + 1.9, t0 + 2.1)])
    oz = clk.summary(2)
    assert oz["samples_in_timed_regions"] == 3
    assert oz["sm_mhz"] == 1455
    assert oz["reasons"] == ["sw_power_cap"]
    assert oz["sm_max_mhz"] == 1965
    dm = clk.summary(1)
    assert dm["samples_in_timed_regions"] == 2 and dm["sm_mhz"] == 1965 and dm["reasons"] == []


def test_all_samples_when_none_inside(tmp_path, monkeypatch):
    t0 = 1_800_000_000.0
    clk = bench.ClockSampler(0)
    clk.path = tmp_path / "clocks.csv"
    clk.path.write_text(_line(t0, 1700, False) + "\n" + _line(t0 + 0.02, 1800, False) + "\n")
    monkeypatch.setattr(bench, "TIMED_WINDOWS", [(2, t0 + 5.0, t0 + 6.0)])
    s = clk.summary(2)
    assert s["samples_in_timed_regions"] == 0 and s["samples"] == 2 and s["sm_mhz"] == 1750


def test_suite_records_each_configuration_and_its_failure(monkeypatch):
    """bench.run_suite: one child process per configuration; a JSON line is kept
    as the result, a non-zero exit or a timeout becomes an error entry and the
    remaining configurations still run."""
    import subprocess

    calls = []

    def fake_run(cmd, capture_output, text, timeout):
        name = cmd[cmd.index("--workload") + 1]
        calls.append((name, cmd[cmd.index("--steps") + 1], cmd[cmd.index("--warmup") + 1]))
        if name == "b":
            return subprocess.CompletedProcess(cmd, 1, "", "CUDA error: out of memory")
        if name == "c":
            raise subprocess.TimeoutExpired(cmd, timeout)
        return subprocess.CompletedProcess(cmd, 0, 'log line\n{"value": 7.5}\n', "")

    monkeypatch.setattr(bench, "SUITE", [("a", "first"), ("b", "second"), ("c", "third")])
    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    out = bench.run_suite(5, 3, timeout_s=9)
    assert [c[0] for c in calls] == ["a", "b", "c"] and calls[0][1:] == ("5", "3")
    assert out["a"]["value"] == 7.5 and "wall_s" in out["a"]
    assert "out of memory" in out["b"]["error"]
    assert out["c"]["error"] == "timed out after 9 s"


def test_suite_entry_is_compacted():
    """compact_entry keeps the figures (value, time, path, errors and checks,
    the U[-1,1] figures) to 4 (errors 3) significant digits and drops the rest."""
    full = {"metric": "SGEMM-SSBTR TFLOP/s", "value": 96.9234567, "unit": "TFLOP/s",
            "ms_per_step": 10.170438385, "full_matrix_tflops": 193.8,
            "rel_err_triangle_vs_double_double": 3.067538308e-08,
            "uniform_inputs": {"value": 107.81835, "ms_per_step": 8.75,
                               "rel_err_triangle_vs_double_double": 2.5299518e-08, "data": "U"},
            "config": {"workload": "psgemm_ssbtr ...", "path": "auto: Ozaki INT8"},
            "n_gpus": 1, "steps": 5, "warmup": 3, "data": "synthetic, seeded",
            "autotune": [{"tile": 0}], "fd_central_h1e-3_plain_max_rel": 8.350186e-08}
    c = bench.compact_entry(full)
    assert c == {"metric": "SGEMM-SSBTR TFLOP/s", "unit": "TFLOP/s", "value": 96.92,
                 "ms_per_step": 10.17, "path": "auto: Ozaki INT8",
                 "rel_err_triangle_vs_double_double": 3.07e-08,
                 "fd_central_h1e-3_plain_max_rel": 8.35e-08,
                 "uniform_inputs": {"value": 107.8, "rel_err": 2.53e-08}}


def test_suite_time_budget(monkeypatch):
    """bench.run_suite: a child gets at most the per-child limit and what is
    left of the suite's budget; once the budget is spent the remaining
    configurations are skipped with a note instead of run."""
    import subprocess

    now = [1000.0]
    limits = []

    def fake_run(cmd, capture_output, text, timeout):
        limits.append(timeout)
        now[0] += 100.0  # every child takes 100 s
        return subprocess.CompletedProcess(cmd, 0, '{"value": 1.0}\n', "")

    monkeypatch.setattr(bench, "SUITE", [(c, c) for c in "abcde"])
    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    monkeypatch.setattr(bench.time, "time", lambda: now[0])
    out = bench.run_suite(5, 3, timeout_s=150, budget_s=305)
    assert limits == [150, 150, 105]
    assert [out[c].get("value") for c in "abc"] == [1.0, 1.0, 1.0]
    assert all("budget" in out[c]["error"] and out[c]["wall_s"] == 0.0 for c in "de")


def test_reference_arm_line_matches_the_headline(tmp_path):
    """`bench.py --impl reference` (the reference library's CPU path on the
    whole headline workload) prints the headline's metric, unit, direction and
    workload, a time per step and the e2e and cpu_baseline objects, so that its
    value and the GPU arm's can be divided."""
    import json
    import os
    import subprocess

    import oracle
    if not oracle.REF_LIB.exists():
        import pytest
        pytest.skip("reference library not built (oracle/_ref)")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, str(Path(bench.__file__)), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       timeout=600, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads([x for x in p.stdout.splitlines() if x.startswith("{")][-1])
    assert line["metric"] == bench.HEADLINE_METRIC and line["unit"] == "TFLOP/s"
    assert line["higher_is_better"] is True and line["impl"] == "reference"
    assert line["config"]["workload"] == bench.workload_name()
    assert line["steps"] == 1 and line["warmup"] == 0 and line["ms_per_step"] > 0
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
