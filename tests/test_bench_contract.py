"""bench.py keeps its one-line JSON contract: the reference arm (the oracle
port on the host cores) on CPU, our arm on the GPU."""
import json
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _run(*args, timeout=600):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True,
                         text=True, timeout=timeout, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference"
    assert d["config"]["workload"].startswith("batched")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


@pytest.mark.gpu
def test_our_arm_line():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = _run("--steps", "3", "--warmup", "3", "--no-cpu-baseline")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "e2e", "gpu_launches", "clocks", "plain_value", "batched_over_plain",
              "every_sweep_schedule", "tuned_plans"):
        assert k in d, k
    r = d["roofline"]
    assert r["bound"] == "int" and 0 < r["frac"] < 2 and r["peak"] > 0
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0
    assert d["gpu_launches"] == 3 * 6 and d["config"]["workload"].startswith("batched")
    assert d["config"]["swap_every"] == 16 and d["config"]["measure_every"] == 1024
    assert d["every_sweep_schedule"]["plain_value"] > 0
