"""Regenerate ref_res_tables.json from the reference's shipped result tables.

The reference (Marco-Mendivil-Carboni/Spin-Glass) ships Simulations/LL/H-res.dat
written by its analyze-all.py: a header line with the total sweep count and
24 rows of 9 columns (beta, chi0, err, xi_L/L, err, e, err, m, err).  These are
its only fixtures.  Usage: python tests/golden/make_ref_tables.py [reference root]
(default: $CSG_REFERENCE_ROOT, else a directory "reference" beside this repository)
"""
import json
import os
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent
root = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else
                    os.environ.get("CSG_REFERENCE_ROOT", str(HERE.parents[2] / "reference")))
out = {}
for f in sorted((root / "Simulations").glob("*/*-res.dat")):
    lines = f.read_text().splitlines()
    rows = [[float(v) for v in ln.split()] for ln in lines[1:] if ln.strip()]
    out[f"{f.parent.name}/{f.name[:-len('-res.dat')]}"] = {
        "source": f"Simulations/{f.parent.name}/{f.name}",
        "header": lines[0],
        "columns": ["beta", "chi0", "chi0_err", "xi_L_over_L", "xi_err", "e", "e_err", "m",
                    "m_err"],
        "rows": rows,
    }
dst = pathlib.Path(__file__).resolve().parent / "ref_res_tables.json"
dst.write_text(json.dumps(out, indent=1) + "\n")
print(dst, len(out), "tables")
