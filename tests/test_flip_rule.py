"""The device acceptance rules (flip_gen for a field, flip_h0 at H = 0) equal
the rule they implement on every spin/bond-count combination, including the
draws at the edges (0, a threshold itself, 0xFFFFFFFF)."""
import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _build(tmp_path):
    exe = tmp_path / "flip_rule_check"
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17",
                    f"-I{ROOT / 'spin-glass_b200' / 'csrc'}", str(ROOT / "tests" / "flip_rule_check.cu"),
                    "-o", str(exe)], check=True, capture_output=True, timeout=600)
    return exe


def test_flip_rule_check_builds(tmp_path):
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_flip_rules_match_the_acceptance_rule(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([str(_build(tmp_path))], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    words = out.stdout.split()
    assert words[0] == "cases" and int(words[1]) > 0
    assert int(words[4]) == 0, out.stdout  # general field
    assert int(words[7]) == 0, out.stdout  # zero field
