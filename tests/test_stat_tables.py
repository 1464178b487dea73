"""The committed statistical-parity results (CPU): every table the reference
ships (Simulations/{12,14,16}/0.0000-res.dat, Simulations/16/{0.0625,0.1250,
0.1875}-res.dat) has a table of this engine beside it, and every entry agrees
within 3 standard errors.

Each table comes twice: `<LL>-<H>-res.dat` with the reference's estimator
(errors from the variance over the 2048 samples, analyze-all.py:37-76) and
`<LL>-<H>-res-word.dat` with the errors taken over the 64 independent words of
32 samples (the samples of a word share their random draws).  The means are
the same in both.  z is recomputed here from the files."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
TABLES = json.loads((GOLD / "ref_res_tables.json").read_text())
COLS = ["beta", "chi0", "chi0_err", "xi", "xi_err", "e", "e_err", "m", "m_err"]
SHIPPED = [(12, 0.0), (14, 0.0), (16, 0.0), (16, 0.0625), (16, 0.125), (16, 0.1875)]


def _ours(L, H, word):
    name = f"{L:02d}-{H:06.4f}-res{'-word' if word else ''}.dat"
    return np.loadtxt(GOLD / "b200_tables" / name)


@pytest.mark.parametrize("L,H", SHIPPED)
def test_table_within_three_sigma(L, H):
    ref = np.array(TABLES[f"{L}/{H:06.4f}"]["rows"])
    per_sample, per_word = _ours(L, H, False), _ours(L, H, True)
    assert per_sample.shape == ref.shape == (24, 9)
    np.testing.assert_allclose(per_sample[:, 0], ref[:, 0], rtol=1e-9)  # same ladder
    for c in ["chi0", "xi", "e", "m"]:
        i, ie = COLS.index(c), COLS.index(c + "_err")
        np.testing.assert_array_equal(per_sample[:, i], per_word[:, i])  # same means
        z = (per_word[:, i] - ref[:, i]) / np.hypot(per_word[:, ie], ref[:, ie])
        assert np.all(np.abs(z) < 3.0), (c, np.round(z, 2))


def test_parity_record_matches_tables():
    rec = {(r["L"], r["H"]): r for r in json.loads((GOLD / "b200_tables" / "stat_parity.json").read_text())}
    assert set(rec) == set(SHIPPED)
    for (L, H), r in rec.items():
        assert r["sweeps"] == 4194304  # the reference's tot_MC_steps
        for c, v in r["compare"].items():
            assert v["n_abs_z_word_gt_3"] == 0
            assert v["max_abs_z_word"] < 3.0
