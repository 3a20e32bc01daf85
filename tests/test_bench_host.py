"""bench.py host logic on the CPU: the reference arm's JSON line and its CPU
time budget, the clock sampler's output shape and the kernel labels."""
import json
import os
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from helix_b200 import systems as S  # noqa: E402


def test_timed_steps_stops_at_the_budget():
    calls = []

    def step():
        calls.append(1)
        time.sleep(0.05)

    n, sec = bench.timed_steps(step, 100, budget_s=0.12)
    assert n == len(calls) and 2 <= n <= 4
    assert sec >= 0.12


def test_timed_steps_runs_every_requested_step_within_budget():
    n, _ = bench.timed_steps(lambda: None, 7, budget_s=10.0)
    assert n == 7


def test_reference_arm_line_for_the_small_config():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["steps"] == 2 and line["steps_requested"] == 2
    assert line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == bench.CONFIGS["c1"]["workload"]
    # our arm builds its config from the same function: the two arms' config objects are identical
    cfg = bench.CONFIGS["c1"]
    assert line["config"] == json.loads(json.dumps(bench.workload_config(cfg, bench.make_problem(cfg), 1)))


def test_clock_sampler_reports_its_fields():
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.1)
    r = c.stop()
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(r)
    assert isinstance(r["reasons"], list)


class _Info:
    def __init__(self, kps):
        self.kernels_per_step = kps


class _Ctx:
    def __init__(self, path, kps=4):
        self.stage_path = path
        self.info = _Info(kps)  # capi.Context keeps the hx_info of its creation (valid after close)


@pytest.mark.parametrize("path,packed,per_stage,want", [
    ("fused", True, 2, "herm_kernel<6> + upterm_kernel per stage (Hermitian-packed slabs)"),
    ("fused", False, 1, "fused_kernel<6> per stage"),
    ("flip", False, 2, "comm_kernel + combine_kernel per stage (spin-flip coupling path)"),
    ("csr", False, 2, "csr_comm_kernel + csr_combine_kernel per stage (general sparse operators)"),
    ("generic", False, 1, "stage_kernel per stage (generic path)"),
    ("small", False, 1, "small_kernel per stage (d <= 16, batched neighbour gathers)"),
])
def test_stage_kernel_labels(path, packed, per_stage, want):
    p = S.spin_glass(6, seed=1, depth=1, K=1)
    assert bench.stage_kernels_label(_Ctx(path), p, packed, per_stage) == want


def test_step_kernel_label():
    p = S.spin_glass(4, seed=1, depth=1, K=1)
    label = bench.stage_kernels_label(_Ctx("small", kps=1), p, False, 1)
    assert label.startswith("small_step_kernel per step")
