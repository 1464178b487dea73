"""Word-blocked errors of spin-glass_b200/analysis.py (CPU).

block = 1 is the reference's estimator (analyze-all.py:37-76); block = b
takes the variance over means of b consecutive samples.  The means never
change; the errors equal std(block means) / sqrt(n_blocks)."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "spin-glass_b200"))
import analysis  # noqa: E402


def _series(tmp_path, n, ndis, nrep, seed=5):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, ndis, nrep), analysis.OBS_DT)
    # a per-block offset shared by the block's samples (correlated noise) plus
    # per-sample noise
    blk = rng.normal(size=(n, ndis // 8, 1, nrep)).repeat(8, axis=1).reshape(n, ndis, nrep)
    for f, k in [("e", 2), ("m", 2)]:
        rec[f] = (blk[..., None] * 0.1 + rng.normal(size=(n, ndis, nrep, k)) * 0.01)
    rec["q_0"] = 0.5 + blk * 0.05 + rng.normal(size=(n, ndis, nrep)) * 0.01
    rec["q_1_r"] = 0.1 + rng.normal(size=(n, ndis, nrep, 3)) * 0.01
    rec["q_1_i"] = 0.1 + rng.normal(size=(n, ndis, nrep, 3)) * 0.01
    path = tmp_path / "x-obs.bin"
    rec.tofile(path)
    return path, rec


def test_block_one_is_reference_estimator(tmp_path):
    path, rec = _series(tmp_path, 6, 64, 4)
    res = analysis.analyze(str(path), 8, 64, 4)
    d = rec[3:]
    e = d["e"].astype(np.float64).mean(axis=(0, 3))
    assert np.allclose(res["e"], e.mean(axis=0))
    assert np.allclose(res["e_err"], np.sqrt(e.var(axis=0) / 64))
    assert res["block"] == 1


def test_block_errors_from_block_means(tmp_path):
    path, rec = _series(tmp_path, 6, 64, 4)
    r1 = analysis.analyze(str(path), 8, 64, 4)
    r8 = analysis.analyze(str(path), 8, 64, 4, block=8)
    for c in ["chi0", "xi", "e", "m"]:
        assert np.allclose(r1[c], r8[c])
    d = rec[3:]
    e = d["e"].astype(np.float64).mean(axis=(0, 3))
    eb = e.reshape(8, 8, 4).mean(axis=1)
    assert np.allclose(r8["e_err"], eb.std(axis=0) / np.sqrt(8))
    q = (d["q_0"].astype(np.float64) ** 2).mean(axis=0).reshape(8, 8, 4).mean(axis=1)
    assert np.allclose(r8["chi0_err"], q.std(axis=0) / np.sqrt(8))
    # the planted per-block noise makes the blocked errors larger
    assert np.all(r8["e_err"] > 2 * r1["e_err"])


def test_block_must_divide_samples(tmp_path):
    path, _ = _series(tmp_path, 4, 64, 4)
    with pytest.raises(ValueError):
        analysis.analyze(str(path), 8, 64, 4, block=5)
