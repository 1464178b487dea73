"""Result tables from `<H>-obs.bin` files, computed in chunks.

Restates the estimators of the reference's analyze-all.py (lines 29-88): drop
the first half of the record series (thermalisation), then per temperature
  chi_0  = [<q_0^2>]                       (disorder average of thermal means)
  xi_L/L = sqrt(chi_0/chi_1 - 1) / (2 sin(pi/L)) / L,  chi_1 from q_1 (3 axes)
  e, m   = [<e>], [<m>]  (thermal mean over measurements and both copies)
with errors from the variance over disorder samples.  Output rows have the
reference's 9 columns (beta, chi0, err, xi_L/L, err, e, err, m, err) in the
same format.  Reads the file in chunks, so tables of multi-GB series fit in a
few hundred MB of memory.

Blocked errors (`block` > 1): the reference's errors treat the NDIS samples as
independent, which they are in its program (every spin of every sample draws
its own random number).  This engine's draws serve the 32 samples of a word
(samples 32w .. 32w+31), so their thermal noise is correlated and the
per-sample variance understates the error where thermal noise dominates the
disorder spread (the energy at high temperature).  With `block` = 32 the
errors come from the variance of the word means over the NDIS/32 words, which
are independent; the means are the same.

  python spin-glass_b200/analysis.py <obs.bin> <L> <NDIS> <NREP> [SBMEAS] [out.dat] [BLOCK]
"""
from __future__ import annotations

import sys

import numpy as np

OBS_DT = np.dtype([("e", "f4", (2,)), ("m", "f4", (2,)), ("q_0", "f4"), ("q_1_r", "f4", (3,)),
                   ("q_1_i", "f4", (3,))])


def _spread(x: np.ndarray, block: int):
    """Disorder mean, variance and error of per-sample values x[ndis, ...]:
    the variance over samples (block 1) or over means of `block` consecutive
    samples, scaled back to one sample (var_block * block), and the error
    sqrt(var / ndis) of the mean in either case."""
    if block <= 1:
        return x.mean(axis=0), x.var(axis=0)
    xb = x.reshape(x.shape[0] // block, block, *x.shape[1:]).mean(axis=1)
    return x.mean(axis=0), xb.var(axis=0) * block


def analyze(path: str, L: int, ndis: int, nrep: int, betas=None, chunk: int = 8,
            block: int = 1) -> dict:
    if block < 1 or ndis % block:
        raise ValueError("block must divide the number of samples")
    size = np.memmap(path, dtype=np.uint8, mode="r").size
    therm = size // 2
    data = np.memmap(path, dtype=OBS_DT, mode="r", offset=therm)
    data = data[: (data.size // (ndis * nrep)) * ndis * nrep].reshape(-1, ndis, nrep)
    n = data.shape[0]
    if n == 0:
        raise ValueError("no records after the thermalisation half")
    s_q0 = np.zeros((ndis, nrep))
    s_qr = np.zeros((ndis, nrep, 3))
    s_qi = np.zeros((ndis, nrep, 3))
    s_e = np.zeros((ndis, nrep))
    s_m = np.zeros((ndis, nrep))
    for a in range(0, n, chunk):
        d = np.asarray(data[a:a + chunk])
        s_q0 += (d["q_0"].astype(np.float64) ** 2).sum(axis=0)
        s_qr += (d["q_1_r"].astype(np.float64) ** 2).sum(axis=0)
        s_qi += (d["q_1_i"].astype(np.float64) ** 2).sum(axis=0)
        s_e += d["e"].astype(np.float64).sum(axis=(0, 3))
        s_m += d["m"].astype(np.float64).sum(axis=(0, 3))
    chi0 = s_q0 / n
    chi0_aa, chi0_v = _spread(chi0, block)
    chi1r, chi1i = s_qr / n, s_qi / n
    (r_a, r_v), (i_a, i_v) = _spread(chi1r, block), _spread(chi1i, block)
    chi1_aa = (r_a + i_a).mean(axis=1)
    chi1_v = (r_v + i_v).mean(axis=1)
    chif = chi0_aa / chi1_aa
    chif_v = chif ** 2 * (chi0_v / chi0_aa ** 2 + chi1_v / chi1_aa ** 2)
    # chif < 1 (hot temperatures, few measurements) gives NaN, as the
    # reference's table does; no warning for that expected case
    with np.errstate(invalid="ignore"):
        xi = np.sqrt(chif - 1) / (2 * np.sin(np.pi / L)) / L
    xi_v = (xi / (2 * (chif - 1))) ** 2 * chif_v
    (e_a, e_v), (m_a, m_v) = _spread(s_e / (2 * n), block), _spread(s_m / (2 * n), block)
    if betas is None:
        betas = np.logspace(1, -3, num=nrep, base=2.0)
    return {"beta": np.asarray(betas), "chi0": chi0_aa, "chi0_err": np.sqrt(chi0_v / ndis),
            "xi": xi, "xi_err": np.sqrt(xi_v / ndis), "e": e_a,
            "e_err": np.sqrt(e_v / ndis), "m": m_a,
            "m_err": np.sqrt(m_v / ndis), "n_meas": n, "block": block}


def analyze_gpu(path: str, L: int, ndis: int, nrep: int, betas=None, device: int = 0) -> dict:
    """analyze() on the GPU (csg_analyze_records): the records after the
    thermalisation half are copied to the device once and reduced there."""
    import ctypes as C

    import torch

    try:
        from . import lib, _check
    except ImportError:  # loaded as a plain module next to the package's __init__
        pkg = sys.modules["spin_glass_b200"]
        lib, _check = pkg.lib, pkg._check
    size = np.memmap(path, dtype=np.uint8, mode="r").size
    data = np.memmap(path, dtype=OBS_DT, mode="r", offset=size // 2)
    n = data.size // (ndis * nrep)
    if n == 0:
        raise ValueError("no records after the thermalisation half")
    host = np.array(data[: n * ndis * nrep]).view(np.float32)  # a writable copy
    dev = torch.from_numpy(host).to(torch.device("cuda", device))
    table = np.zeros((nrep, 8), np.float64)
    _check(lib().csg_analyze_records(C.c_void_p(dev.data_ptr()), n, ndis, nrep, L,
                                     table.ctypes.data_as(C.c_void_p), None))
    if betas is None:
        betas = np.logspace(1, -3, num=nrep, base=2.0)
    cols = ["chi0", "chi0_err", "xi", "xi_err", "e", "e_err", "m", "m_err"]
    res = {"beta": np.asarray(betas), "n_meas": n}
    res.update({c: table[:, k] for k, c in enumerate(cols)})
    return res


def write_table(res: dict, path: str, sweeps_per_meas: int = 1024) -> None:
    with open(path, "w") as f:
        f.write(f"# tot_MC_steps : {2 * res['n_meas'] * sweeps_per_meas:,}\n")
        cols = ["beta", "chi0", "chi0_err", "xi", "xi_err", "e", "e_err", "m", "m_err"]
        for r in range(len(res["beta"])):
            f.write("".join(f"{res[c][r]:16.12f}" for c in cols) + "\n")


if __name__ == "__main__":
    obs, L, ndis, nrep = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4])
    sbmeas = int(sys.argv[5]) if len(sys.argv) > 5 else 1024
    out = sys.argv[6] if len(sys.argv) > 6 else obs.replace("-obs.bin", "-res.dat")
    block = int(sys.argv[7]) if len(sys.argv) > 7 else 1
    write_table(analyze(obs, L, ndis, nrep, block=block), out, sbmeas)
    print(out)
