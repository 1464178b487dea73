"""Record the reference program's own outputs as small test fixtures.

Runs the reference's CUDA program once from a fresh start on a GPU, in a
scratch directory, and keeps a slice of the two files it writes.  The program
is built from the reference's own sources by `oracle/build_ref.sh <root> <L>
<SPFILE>` (only the compile-time L and SPFILE change), e.g. into
oracle/_ref/csg_ref_L8_S2048.

Kept (for the first n_samples disorder samples):
  * chkpt: `<H>-chkpt.bin`, the lattice array after the run — lattice
    2*sample+copy, site (z*L+y)*L+x, bits 0..23 the spins by temperature
    (eamsim.cu:655-662, written after `rearrange`, :419-448, put the
    temperatures in order), bits 26..31 the bonds;
  * obs: the last record block of `<H>-obs.bin` (obs_s [NDIS][NREP],
    eamsim.cu:703-707).  Its q_0 / q_1 fields come from `compute_q` on that
    same lattice (eamsim.cu:698-701); its e / m fields come from the last
    exchange round, 16 sweeps earlier (eamsim.cu:388, 407-415).

The reference seeds its generators from the clock (eamsim.cu:539, 627), so
every run gives other numbers; the fixture is one such run, kept as it came.

Usage: python tests/golden/make_ref_run_fixtures.py <out dir> <program> <L> <n_samples> [H]
"""
from __future__ import annotations

import json
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

NDIS, NCP, NREP = 2048, 2, 24  # eamsim.cuh:16-17, 25 (unchanged by build_ref.sh)


def main() -> None:
    out_dir = pathlib.Path(sys.argv[1])
    prog = pathlib.Path(sys.argv[2]).resolve()
    L, ns = int(sys.argv[3]), int(sys.argv[4])
    H = float(sys.argv[5]) if len(sys.argv) > 5 else 0.0
    N = L ** 3
    out_dir.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        r = subprocess.run([str(prog), td, repr(H)], cwd=td, capture_output=True, text=True,
                           timeout=600)
        if r.returncode != 0:
            raise SystemExit(f"reference program failed ({r.returncode}): {r.stdout}{r.stderr}")
        stem = f"{H:06.4f}"
        chk = np.fromfile(pathlib.Path(td) / f"{stem}-chkpt.bin", dtype=np.uint32)
        obs = np.fromfile(pathlib.Path(td) / f"{stem}-obs.bin", dtype=np.float32)
    assert chk.size == NDIS * NCP * N, chk.size
    blocks = obs.size // (NDIS * NREP * 11)
    assert obs.size == blocks * NDIS * NREP * 11 and blocks >= 1
    last = obs.reshape(blocks, NDIS, NREP, 11)[-1]
    dst = out_dir / f"ref_run_L{L}.npz"
    np.savez_compressed(
        dst, chkpt=chk.reshape(NDIS * NCP, N)[: NCP * ns].copy(), obs=last[:ns].copy(),
        meta=np.array(json.dumps({"L": L, "H": H, "n_samples": ns, "ndis_run": NDIS,
                                  "record_blocks": blocks, "program": prog.name,
                                  "stdout": r.stdout[-400:]})))
    print(dst, "blocks", blocks)


if __name__ == "__main__":
    main()
