"""Statistical parity with the reference's result tables (needs a GPU; slow).

Runs the `csg` command with the reference's production settings (NDIS=2048,
NCP=2, NREP=24, SBSHFL=16, SBMEAS=1024, SPFILE=262144, 16 chained invocations =
4,194,304 sweeps, beta ladder 2 (2^(-4/23))^r) for the lattices and fields of
the shipped tables Simulations/{12,14,16}/<H>-res.dat, reduces each series with
spin-glass_b200/analysis.py, and compares every entry with the shipped value:
z = (ours - ref) / sqrt(err_ours^2 + err_ref^2), once with the reference's
per-sample errors on both sides ("z") and once with this engine's errors taken
over the 64 independent words of 32 samples ("z_word"; the 32 samples of a
word share their random draws, so their thermal noise is correlated).

  python tests/stat_parity.py <out_dir> [n_files] [L:H ...]

Writes <out_dir>/<LL>-<H>-res.dat and <out_dir>/stat_parity.json.  The series
files (8.8 GB each at 16 files) are written under $CSG_STAT_WORK (default:
<out_dir>) and deleted after each reduction.  Seeds: 20240000 + L at H = 0,
plus 100 * round(10000 H) at H != 0 (independent disorder per table), plus
$CSG_STAT_SEED_OFFSET (default 0) for a repeat with other disorder.
"""
from __future__ import annotations

import json
import os
import pathlib
import shutil
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "spin-glass_b200"))
import analysis  # noqa: E402

CLI = ROOT / "spin-glass_b200" / "csg"
TABLES = json.loads((ROOT / "tests" / "golden" / "ref_res_tables.json").read_text())
COLS = ["beta", "chi0", "chi0_err", "xi", "xi_err", "e", "e_err", "m", "m_err"]


def run_case(out: pathlib.Path, L: int, H: float, n_files: int, seed: int) -> dict:
    work = pathlib.Path(os.environ.get("CSG_STAT_WORK", str(out)))
    d = work / f"sim-{L:02d}-{H:06.4f}"
    d.mkdir(parents=True, exist_ok=True)
    (d / "csg.conf").write_text(f"L = {L}\nseed = {seed}\n")
    t0 = time.time()
    for k in range(n_files):
        r = subprocess.run([str(CLI), str(d), f"{H}"], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stdout + r.stderr)
    wall = time.time() - t0
    obs = d / f"{H:06.4f}-obs.bin"
    res = analysis.analyze(str(obs), L, 2048, 24)
    res_w = analysis.analyze(str(obs), L, 2048, 24, block=32)
    table = out / f"{L:02d}-{H:06.4f}-res.dat"
    analysis.write_table(res, str(table))
    analysis.write_table(res_w, str(out / f"{L:02d}-{H:06.4f}-res-word.dat"))
    shutil.rmtree(d)
    ref = TABLES.get(f"{L}/{H:06.4f}")
    cmp = {}
    if ref is not None:
        rows = np.array(ref["rows"])
        for c, ce in [("chi0", "chi0_err"), ("xi", "xi_err"), ("e", "e_err"), ("m", "m_err")]:
            i, ie = COLS.index(c), COLS.index(ce)
            z = (res[c] - rows[:, i]) / np.sqrt(res[ce] ** 2 + rows[:, ie] ** 2)
            zw = (res[c] - rows[:, i]) / np.sqrt(res_w[ce] ** 2 + rows[:, ie] ** 2)
            cmp[c] = {"max_abs_z": float(np.nanmax(np.abs(z))),
                      "n_abs_z_gt_3": int(np.sum(np.abs(z) > 3)),
                      "z": [round(float(v), 2) for v in z],
                      "max_abs_z_word": float(np.nanmax(np.abs(zw))),
                      "n_abs_z_word_gt_3": int(np.sum(np.abs(zw) > 3)),
                      "err_ratio_word": [round(float(v), 2) for v in res_w[ce] / res[ce]],
                      "z_word": [round(float(v), 2) for v in zw]}
    return {"L": L, "H": H, "files": n_files, "sweeps": n_files * 262144, "wall_s": round(wall, 1),
            "table": table.name, "compare": cmp}


def main() -> None:
    out = pathlib.Path(sys.argv[1])
    out.mkdir(parents=True, exist_ok=True)
    n_files = int(sys.argv[2]) if len(sys.argv) > 2 else 16
    cases = [tuple(a.split(":")) for a in sys.argv[3:]] or [("12", "0"), ("14", "0"), ("16", "0"),
                                                             ("16", "0.1875")]
    results = []
    for L, H in cases:
        seed = (20240000 + int(L) + 100 * int(round(10000 * float(H))) +
                int(os.environ.get("CSG_STAT_SEED_OFFSET", "0")))
        results.append(run_case(out, int(L), float(H), n_files, seed=seed))
        (out / "stat_parity.json").write_text(json.dumps(results, indent=1))
        r = results[-1]
        print(r["L"], r["H"], r["wall_s"],
              {k: (round(v["max_abs_z"], 2), v["n_abs_z_gt_3"], round(v["max_abs_z_word"], 2),
                   v["n_abs_z_word_gt_3"]) for k, v in r["compare"].items()}, flush=True)


if __name__ == "__main__":
    main()
