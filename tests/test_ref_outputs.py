"""Parity with the reference program's own outputs.

The fixtures under tests/golden/ref_run/ were written by the reference's CUDA
program itself (Program/src, built from its sources with only L and SPFILE
changed, run once on a B200 by tests/golden/make_ref_run_fixtures.py): the
checkpoint it saved after a 2048-sweep run (lattice 2*sample+copy, bits 0..23
spins by temperature after `rearrange`, bits 26..31 bonds; eamsim.cu:655-662)
and the last block of observable records it appended (eamsim.cu:703-707),
sliced to the first samples.  The q_0 / q_1 fields of that block come from
`compute_q` (eamsim.cu:451-511) on that same checkpointed lattice, so they are
a deterministic function of the fixture's state.  The e / m fields are not:
they are the energies of the last exchange round, 16 sweeps before the saved
state (eamsim.cu:388, 407-415), and are not compared.

Bars: q_0 bit-exact (the reference sums +-1 in float, exact below 2^24, then
divides by N); q_1 within 1e-6 absolute (the reference accumulates
l_q*cosf(k*x) in float over the sites, the engine and the oracle form the
same sums from exact integer counts in double).
"""
import json
import pathlib

import numpy as np
import pytest

from oracle import refdefs

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ref_run"
CASES = [8, 12]
Q1_ATOL = 1e-6


def load_case(L: int):
    z = np.load(GOLDEN / f"ref_run_L{L}.npz")
    meta = json.loads(str(z["meta"]))
    assert meta["L"] == L and meta["ndis_run"] == 2048
    return z["chkpt"], z["obs"], meta


@pytest.mark.parametrize("L", CASES)
def test_reference_checkpoint_layout(L):
    """The reference's checkpoint follows the layout the engine reads: the two
    copies of a sample carry the same bond bits, and each bond is stored at
    both of its ends (eamsim.cu:598-616, 634-641)."""
    chk, obs, meta = load_case(L)
    ns = meta["n_samples"]
    assert chk.shape == (2 * ns, L ** 3) and obs.shape == (ns, 24, 11)
    for s in range(ns):
        assert np.array_equal(chk[2 * s] >> 26, chk[2 * s + 1] >> 26)
        assert refdefs.bond_bits_consistent(chk[2 * s], L)
    assert np.all((chk & np.uint32(0x03000000)) == 0), "bits 24, 25 are unused"


@pytest.mark.parametrize("L", CASES)
def test_restated_compute_q_matches_reference_output(L):
    """oracle/refdefs.py's compute_q on the reference's checkpoint reproduces
    the reference's own q_0 / q_1 records."""
    chk, obs, meta = load_case(L)
    for s in range(meta["n_samples"]):
        q0, qr, qi = refdefs.overlaps(chk[2 * s], chk[2 * s + 1], L, 24)
        assert np.array_equal(q0.astype(np.float32), obs[s, :, 4])
        np.testing.assert_allclose(qr, obs[s, :, 5:8], rtol=0, atol=Q1_ATOL)
        np.testing.assert_allclose(qi, obs[s, :, 8:11], rtol=0, atol=Q1_ATOL)


@pytest.mark.parametrize("L", CASES)
def test_oracle_reads_reference_checkpoint(orc, L):
    """The oracle converts the reference's checkpoint to the engine layout and
    back without loss, and its records of that state reproduce the
    reference's q_0 exactly and q_1 within the bar."""
    chk, obs, meta = load_case(L)
    spins, bonds = orc.from_ref_lattice(chk, L, 24)
    assert np.array_equal(orc.to_ref_lattice(spins, bonds, L), chk)
    rec = orc.obs_records(spins, bonds, L, meta["H"])
    assert np.array_equal(rec[:, :, 4], obs[:, :, 4])
    np.testing.assert_allclose(rec[:, :, 5:11], obs[:, :, 5:11], rtol=0, atol=Q1_ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("L", CASES)
def test_engine_resumes_reference_checkpoint(csg, orc, L):
    """The drop-in resume path (main.cu:40-54): csg_load_checkpoint accepts the
    reference's own checkpoint, csg_save_checkpoint gives it back byte for
    byte, and csg_obs_records of that state reproduces the q_0 / q_1 records
    the reference wrote for it."""
    chk, obs, meta = load_case(L)
    W = meta["n_samples"] // 32
    betas = csg.reference_betas(24)
    with csg.Engine(L, W, 2, betas, H=meta["H"], seed=7, sweeps_per_swap=16,
                    sweeps_per_meas=1024) as e:
        e.load_checkpoint(chk, 0)
        assert np.array_equal(e.save_checkpoint(), chk)
        spins, bonds, _ = e.get_state()
        ospins, obonds = orc.from_ref_lattice(chk, L, 24)
        assert np.array_equal(spins, ospins) and np.array_equal(bonds, obonds)
        rec = e.obs_records()
    assert np.array_equal(rec[:, :, 4], obs[:, :, 4])
    np.testing.assert_allclose(rec[:, :, 5:11], obs[:, :, 5:11], rtol=0, atol=Q1_ATOL)
