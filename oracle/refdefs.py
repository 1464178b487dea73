"""Restatement, in numpy, of the reference's own measurement definitions on its
own packed lattice layout (test infrastructure only).

The reference (Program/src of Marco-Mendivil-Carboni/Spin-Glass) keeps one
uint32 per site per lattice: bits 0..23 the spins of 24 temperatures, bits
26..31 the six bonds of the site (eamsim.cuh:27-35).  These functions follow
its code path literally — the sublattice it sums over, its satisfied-bond
counting through ``J ^ n ^ c`` and its float formulas — so the oracle's
sample-packed energies, magnetisations and overlaps can be checked against the
reference's definitions, not against a second copy of the oracle.
"""
from __future__ import annotations

import numpy as np

SHIFTSJ = 26  # eamsim.cuh:35


def _coords(L: int):
    i = np.arange(L ** 3)
    return i % L, (i // L) % L, i // (L * L)


def _neighbours(L: int):
    """Site indices of the 6 neighbours in the reference's order
    (eamsim.cu:155-161: x-1, x+1, y-1, y+1, z-1, z+1)."""
    x, y, z = _coords(L)

    def idx(xx, yy, zz):
        return (L * L * (zz % L) + L * (yy % L) + (xx % L)).astype(np.int64)

    return [idx(x - 1, y, z), idx(x + 1, y, z), idx(x, y - 1, z), idx(x, y + 1, z),
            idx(x, y, z - 1), idx(x, y, z + 1)]


def energy_magnetization(lattice: np.ndarray, L: int, H: float, nrep: int):
    """perform_PT_shuffle (eamsim.cu:237-325) for one lattice uint32[N]:
    returns float32 arrays e[nrep] (total energy, eamsim.cu:324) and
    m[nrep] (total magnetisation, eamsim.cu:323)."""
    lat = lattice.astype(np.uint64)
    x, y, z = _coords(L)
    # the threads of perform_PT_shuffle sit on x = 2*tx + ((z&1)^(y&1)),
    # i.e. on the sites with x+y+z even (eamsim.cu:238-249)
    sub = ((x + y + z) % 2) == 0
    nb = _neighbours(L)
    c = lat[sub]
    sat = np.zeros(nrep, np.int64)
    for k in range(6):
        jmask = np.where((c >> np.uint64(SHIFTSJ + k)) & np.uint64(1), np.uint64(0xFFFFFFFF),
                         np.uint64(0))
        inter = jmask ^ lat[nb[k][sub]] ^ c  # eamsim.cu:260-265
        for r in range(nrep):
            sat[r] += int(((inter >> np.uint64(r)) & np.uint64(1)).sum())
    ups = np.array([int(((lat >> np.uint64(r)) & np.uint64(1)).sum()) for r in range(nrep)])
    N = L ** 3
    e = np.float32(2) * sat.astype(np.float32) - np.float32(6 * (N // 2))  # eamsim.cu:322
    m = np.float32(2) * ups.astype(np.float32) - np.float32(N)             # eamsim.cu:323
    e = -(e + np.float32(H) * m)                                            # eamsim.cu:324
    return e.astype(np.float32), m.astype(np.float32)


def overlaps(lat0: np.ndarray, lat1: np.ndarray, L: int, nrep: int):
    """compute_q (eamsim.cu:451-511) for the two copies of one sample:
    q_0[nrep], q_1_r[nrep,3], q_1_i[nrep,3] (float64 sums of the same terms)."""
    x, y, z = _coords(L)
    N = L ** 3
    k = 2 * np.pi / L
    q0 = np.zeros(nrep)
    qr = np.zeros((nrep, 3))
    qi = np.zeros((nrep, 3))
    for r in range(nrep):
        s0 = 2 * ((lat0 >> r) & 1).astype(np.int64) - 1
        s1 = 2 * ((lat1 >> r) & 1).astype(np.int64) - 1
        lq = (s0 * s1).astype(np.float64)
        q0[r] = lq.sum() / N
        for d, co in enumerate((x, y, z)):
            qr[r, d] = (lq * np.cos(k * co)).sum() / N
            qi[r, d] = (lq * np.sin(k * co)).sum() / N
    return q0, qr, qi


def bond_bits_consistent(lattice: np.ndarray, L: int) -> bool:
    """The reference stores each bond at both of its ends (eamsim.cu:598-616):
    bit 26+2d of a site equals bit 27+2d of its -d neighbour."""
    nb = _neighbours(L)
    lat = lattice.astype(np.uint64)
    for d in range(3):
        minus = (lat >> np.uint64(SHIFTSJ + 2 * d)) & np.uint64(1)
        plus_of_nb = (lat[nb[2 * d]] >> np.uint64(SHIFTSJ + 2 * d + 1)) & np.uint64(1)
        if not np.array_equal(minus, plus_of_nb):
            return False
    return True


def prob_table(beta: float, H: float) -> np.ndarray:
    """compute_prob (eamsim.cu:24-40) for one temperature, in float32 as the
    reference does it: entry i = 2c+b (c satisfied bonds, b centre bit) is
    expf(2*beta*E_i)*UINT_MAX with E_i = -(i-6-H-(1-2H)(i&1)); entries 14, 15
    keep the initial value UINT_MAX (eamsim.cu:8-21).  Returned as float64 of
    the float32 product (the uint64 cast of the reference saturates above
    2^64 and is only compared against 32-bit draws)."""
    out = np.full(16, np.float64(np.float32(4294967295.0)))
    for i in range(14):
        energy = np.float32(-(i - 6 - H - ((1 - 2 * H) * (i & 1))))
        out[i] = np.float64(np.float32(np.exp(np.float32(beta) * np.float32(2) * energy,
                                              dtype=np.float32)) * np.float32(4294967295.0))
    return out
