"""The benchmark script's CPU-side contract (no GPU needed).

* ``sample_blocks``: the CPU baseline's step blocks lie inside the span, do
  not overlap and are spread over it, any prefix too.
* ``bench.py --impl reference``: the reference arm (the CPU restatement of
  the reference algorithm) prints one JSON line with the metric, unit and
  config of the GPU arm, ``impl: "reference"``, a ``cpu_baseline`` that
  describes the run and an ``e2e`` equal to its value with no transfers.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


@pytest.mark.parametrize("n_steps,block,n_blocks", [(480, 16, 30), (480, 16, 5), (3360, 16, 12), (48, 16, 8),
                                                     (20, 16, 4)])
def test_sample_blocks_spread_inside_the_span(n_steps, block, n_blocks):
    starts = bench.sample_blocks(n_steps, block, n_blocks)
    assert 1 <= len(starts) <= max(1, n_steps // block)
    assert all(0 <= s and s + block <= n_steps for s in starts)
    srt = sorted(starts)
    assert all(b - a >= block for a, b in zip(srt, srt[1:]))  # no overlap
    if len(starts) >= 2:
        # The first two blocks already come from both halves of the span.
        half = n_steps / 2
        assert min(starts[:2]) < half <= max(starts[:2]) + block


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    from mizuba_b200 import synth

    assert d["config"] == bench.workload_config(synth.workload("c2_20k_1d"))
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
