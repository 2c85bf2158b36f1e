"""The benchmark's own arm on the GPU: one JSON line with the keys its consumers read (metric, the
device-timed value, the end-to-end figure with its copies, the dominant kernel's roofline with its
traffic, the clocks sampled during the timed frames and the count of the library's launches)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_contract():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--small", "--steps", "1", "--warmup", "3",
                        "--no-extras"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [s for s in r.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    import bench

    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is False
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    assert line["value"] > 0 and line["ms_per_step"] == line["value"]
    assert line["scaling"] == "weak" and line["vs_baseline"] is None and line["data"] == "synthetic"
    assert line["config"]["workload"] and line["config"]["method"] == "learned"
    e2e = line["e2e"]
    assert e2e["value"] >= line["value"] * 0.9 and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    roof = line["roofline"]
    assert roof["kernel"] == "learned_level" and roof["bound"] == "tensor" and roof["unit"] == "TFLOP/s"
    assert 0 < roof["frac"] < 1.5 and roof["achieved"] == pytest.approx(roof["frac"] * roof["peak"])
    assert roof["traffic"] > 0 and roof["rows_per_frame"] > 0
    assert line["cut_eval_roofline"]["frac"] > 0
    assert line["gpu_launches"] > 0 and line["launches_per_frame"] > 0
    clk = line["clocks"]
    assert clk["sm_max_mhz"] is None or clk["sm_max_mhz"] > 0
    assert isinstance(clk["reasons"], list)
    for stage in ("cut_learned", "cut_lists", "cut_eval"):
        assert line["stage_ms"][stage] > 0
