"""Pins of the CPU oracle against published vectors and the reference's own
definitions and fixtures (no GPU)."""
import json
import pathlib

import numpy as np
import pytest

from oracle import refdefs

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# Philox4x32-10 known-answer vectors published with Random123 (kat_vectors).
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers(orc, ctr, key, expect):
    assert [int(v) for v in orc.philox(ctr, key)] == expect


@pytest.mark.parametrize("H", [0.0, 0.0625, 0.1875, 1.0, 2.5])
def test_thresholds_match_reference_prob_table(orc, H):
    """thr[t][s][U] is the reference's s_prob[2c+s] (c = 6-U satisfied bonds)
    computed in double instead of float32 (eamsim.cu:24-40)."""
    betas = orc.reference_betas(24)
    thr = orc.thresholds(betas, H)
    for t, beta in enumerate(betas):
        ref = refdefs.prob_table(beta, H)
        for s in (0, 1):
            for U in range(7):
                ours = int(thr[t, s, U])
                r = ref[2 * (6 - U) + s]
                if ours == 1 << 32:
                    assert r >= 4294967295.0 * (1 - 1e-6)
                else:
                    assert abs(ours - r) <= 4e-6 * max(r, 1.0) + 1.0, (t, s, U, ours, r)


def test_thresholds_monotone_and_h0_shape(orc):
    thr = orc.thresholds(orc.geometric_betas(16, 0.2, 2.0), 0.0)
    assert (np.diff(thr.astype(np.float64), axis=2) >= 0).all()
    assert (thr[:, :, 3:] == 1 << 32).all()
    assert (thr[:, 0, :] == thr[:, 1, :]).all()


def test_init_is_deterministic_and_unbiased(orc):
    s1, b1 = orc.init(8, 2, 2, 8, 99)
    s2, b2 = orc.init(8, 2, 2, 8, 99)
    s3, _ = orc.init(8, 2, 2, 8, 100)
    assert np.array_equal(s1, s2) and np.array_equal(b1, b2)
    assert not np.array_equal(s1, s3)
    frac = np.unpackbits(b1.view(np.uint8)).mean()
    assert abs(frac - 0.5) < 0.01


@pytest.mark.parametrize("L,T,H", [(4, 8, 0.0), (6, 24, 0.1875), (8, 12, 1.5)])
def test_energies_match_reference_definition(orc, L, T, H):
    """Oracle energies/magnetisations == perform_PT_shuffle's (eamsim.cu:237-325)
    evaluated on the same state in the reference's packed layout."""
    spins, bonds = orc.init(L, 1, 2, T, 7)
    betas = orc.geometric_betas(T, 0.5, 2.0)
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=7, sweep0=0, n_sweeps=5)
    ref = orc.to_ref_lattice(spins, bonds, L)
    e, m = orc.energies(spins, bonds, L)
    for n in (0, 5, 31):
        for c in (0, 1):
            re, rm = refdefs.energy_magnetization(ref[2 * n + c], L, H, T)
            ours_e = -(np.float32(-e[0, c, :, n]) + np.float32(H) * m[0, c, :, n].astype(np.float32))
            assert np.array_equal(rm, m[0, c, :, n].astype(np.float32))
            assert np.array_equal(re, ours_e.astype(np.float32))


@pytest.mark.parametrize("L,T", [(4, 8), (6, 12)])
def test_obs_records_match_reference_compute_q(orc, L, T):
    spins, bonds = orc.init(L, 1, 2, T, 11)
    orc.run(spins, bonds, L=L, betas=orc.geometric_betas(T, 0.5, 2.0), H=0.0, seed=11,
            sweep0=0, n_sweeps=3)
    rec = orc.obs_records(spins, bonds, L, 0.0)
    ref = orc.to_ref_lattice(spins, bonds, L)
    for n in (0, 17):
        q0, qr, qi = refdefs.overlaps(ref[2 * n], ref[2 * n + 1], L, T)
        np.testing.assert_array_equal(rec[n, :, 4], q0.astype(np.float32))
        np.testing.assert_allclose(rec[n, :, 5:8], qr, atol=2e-6)
        np.testing.assert_allclose(rec[n, :, 8:11], qi, atol=2e-6)


def test_reference_lattice_round_trip(orc):
    spins, bonds = orc.init(6, 2, 2, 24, 3)
    ref = orc.to_ref_lattice(spins, bonds, 6)
    assert all(refdefs.bond_bits_consistent(ref[i], 6) for i in range(0, 128, 13))
    s2, b2 = orc.from_ref_lattice(ref, 6, 24)
    assert np.array_equal(s2, spins) and np.array_equal(b2, bonds)
    bad = ref.copy()
    bad[1, 0] ^= 1 << 27  # copy 1 disagrees with copy 0 on a bond
    with pytest.raises(RuntimeError):
        orc.from_ref_lattice(bad, 6, 24)


def test_exchange_preserves_configurations(orc):
    """An exchange only permutes configurations between planes: the multiset
    of per-sample energies over temperatures is unchanged by the swap step."""
    L, T = 6, 8
    spins, bonds = orc.init(L, 1, 1, T, 5)
    betas = orc.geometric_betas(T, 0.5, 2.0)
    obs = orc.Observables(L, 1, 1, T, log_rounds=20)
    orc.run(spins, bonds, L=L, betas=betas, H=0.0, seed=5, sweep0=0, n_sweeps=20,
            sweeps_per_swap=1, obs=obs)
    assert obs.swap_rounds == 20 and obs.boundary == 0
    assert obs.swap_log[:20].any()
    assert obs.swap_log[0::2, ..., 1::2].sum() == 0  # even rounds never pair (odd, even)
    assert obs.swap_log[1::2, ..., 0::2].sum() == 0  # odd rounds never pair (even, odd)


def _ref_tables():
    return json.loads((GOLDEN / "ref_res_tables.json").read_text())


def test_high_temperature_energy_matches_reference_table(orc):
    """The shipped L=16 table (Simulations/16/0.0000-res.dat) at the two
    hottest temperatures vs a short oracle run at L=8 (finite-size effects are
    far below the tolerance at these temperatures)."""
    tab = _ref_tables()["16/0.0000"]
    rows = tab["rows"][-2:]
    betas = np.array([r[0] for r in rows] * 2)  # 4 planes
    L, W = 8, 2
    spins, bonds = orc.init(L, W, 2, 4, 2024)
    obs = orc.Observables(L, W, 2, 4)
    orc.run(spins, bonds, L=L, betas=betas, H=0.0, seed=2024, sweep0=0, n_sweeps=300,
            sweeps_per_swap=0, sweeps_per_meas=1, meas_start=100, obs=obs)
    N = L ** 3
    e = obs.e_sum / (obs.n_meas * N)  # [W, C, T, 32]
    for k, r in enumerate(rows):
        per_sample = e[:, :, [k, k + 2], :].mean(axis=(1, 2)).ravel()
        mean, err = per_sample.mean(), per_sample.std(ddof=1) / np.sqrt(per_sample.size)
        assert abs(mean - r[5]) < 5 * err + 1e-4, (r[0], mean, r[5], err)


_OBS_FIELDS = ("e_sum", "m_sum", "q_sum", "q2_sum", "q4_sum", "hist", "e_last", "m_last",
               "d_last", "swap_acc", "swap_log")


@pytest.mark.parametrize("L,W,C_,T,H,sps,spm,word0", [
    (4, 1, 2, 4, 0.0, 1, 1, 0),
    (6, 2, 2, 8, 0.1875, 1, 1, 3),
    (8, 1, 1, 12, 1.5, 2, 3, 0),
    (10, 1, 2, 8, 2.5, 1, 2, 0),
    (12, 1, 2, 16, 4.0, 16, 1024, 7),
])
def test_multispin_run_equals_the_per_sample_restatement(orc, L, W, C_, T, H, sps, spm, word0):
    """orc_run_multispin (the CPU timing baseline: all 32 samples of a word at
    once) gives the per-sample restatement's bits: spins and every
    observable, with exchanges and measurements, at zero and non-zero field."""
    betas = orc.geometric_betas(T, 0.3, 2.0)
    n = 24
    out = []
    for multispin in (False, True):
        spins, bonds = orc.init(L, W, C_, T, 99 + L, word0)
        obs = orc.Observables(L, W, C_, T, log_rounds=n)
        orc.run(spins, bonds, L=L, betas=betas, H=H, seed=99 + L, sweep0=5, n_sweeps=n,
                sweeps_per_swap=sps, sweeps_per_meas=spm, obs=obs, word0=word0,
                multispin=multispin)
        out.append((spins, obs))
    (s0, o0), (s1, o1) = out
    np.testing.assert_array_equal(s1, s0)
    for f in _OBS_FIELDS:
        np.testing.assert_array_equal(getattr(o1, f), getattr(o0, f), err_msg=f)
    assert (o1.n_meas, o1.swap_rounds, o1.boundary) == (o0.n_meas, o0.swap_rounds, o0.boundary)
    assert o0.n_meas > 0 or spm > n
