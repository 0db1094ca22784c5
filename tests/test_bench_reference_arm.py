"""The reference arm of bench.py (`--impl reference`) on the host cores: its JSON line reports the
steps it actually timed, marks a step whose walk ran out of budget as extrapolated, and its
per-step time is the sum of the measured pieces (PM and build unscaled, only the walk scaled by
target count).  Runs the reference's CPU code compiled from its sources (oracle/_ref), so it is
skipped where that library was not built."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

N64 = 64 ** 3


def _ref_available():
    from oracle import oracle as O

    return O.ref_available()


def _run(budget, steps, extra_env=None):
    env = dict(os.environ, BZ_REFERENCE_BUDGET_S=str(budget), OMP_NUM_THREADS="4")
    env.update(extra_env or {})
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "treepm64",
                          "--steps", str(steps), "--warmup", "3"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    return [json.loads(ln) for ln in lines]


def _step_s(line):
    p = line["cpu_baseline"]["pieces"]
    return p["pm_s"] + p["build_s"] + p["walk_s"] * N64 / p["walk_targets"]


@pytest.mark.skipif(not _ref_available(), reason="reference CPU library not built")
def test_reference_arm_reports_the_steps_it_timed():
    (line,) = _run(120, 2)
    assert line["impl"] == "reference" and line["config"]["particles"] == N64
    assert 1 <= line["steps"] <= line["steps_requested"] == 2
    assert line["extrapolated"] is False and line["cpu_baseline"]["extrapolated"] is False
    assert line["cpu_baseline"]["pieces"]["walk_targets"] == N64
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    # the whole run's measured time covers every step it reports
    assert line["measured_s"] >= line["steps"] * 0.5 * line["ms_per_step"] / 1e3
    if line["steps"] == 1:
        assert line["ms_per_step"] == pytest.approx(1e3 * _step_s(line), rel=1e-9)


@pytest.mark.skipif(not _ref_available(), reason="reference CPU library not built")
def test_reference_arm_marks_a_budget_cut_walk_as_extrapolated():
    (line,) = _run(0.05, 4)
    # the PM and the build run in full once; the walk stops after its first chunk
    assert line["steps"] == 1 and line["extrapolated"] is True
    pieces = line["cpu_baseline"]["pieces"]
    assert 0 < pieces["walk_targets"] < N64
    assert line["ms_per_step"] == pytest.approx(1e3 * _step_s(line), rel=1e-9)
    assert "scaled to all" in line["cpu_baseline"]["sample"]


def test_reference_arm_other_ranks_exit_without_work():
    lines = _run(0.05, 1, {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert lines == []
