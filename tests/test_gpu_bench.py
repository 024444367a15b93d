"""bench.py keeps its output contract: one JSON line with the metric, the
device-timed value, the PCG rooflines (L2 at the benchmark size, HBM on the
larger case), the end-to-end number through the C ABI, the launch count and
the extension keys (multigrid, two-level, batch)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_contract():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "3", "--warmup", "3",
                        "--e2e-steps", "2", "--no-cpu-baseline", "--precision", "fp64", "--hbm-n", "24",
                        "--hbm-steps", "1", "--batch-steps", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["config"]["workload"].startswith("lid-driven cavity 64^3")
    roof = d["roofline"]
    assert roof["bound"] == "l2" and roof["unit"] == "GB/s" and roof["achieved"] > 0
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-9
    assert roof["kernel_bytes_per_iteration"] > 0 and roof["allreduce_us"] > 0
    hbm = d["hbm_case"]
    assert hbm["bound"] == "hbm" and hbm["achieved"] > 0 and abs(hbm["frac"] - hbm["achieved"] / hbm["peak"]) < 1e-9
    # a fraction above ~1 would mean the byte model overstates what the kernel moves
    for r in (roof, hbm, d["multigrid"]["roofline"]):
        assert 0.0 < r["frac"] <= 1.2, r
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    assert d["two_level"]["value"] > 0
    assert d["multigrid"]["value"] > 0 and d["multigrid"]["pcg_kernel"] == 7
    assert d["batch"]["fp64"]["value"] > 0 and d["batch"]["mixed"]["value"] > 0
