"""Bit-exact parity with the CPU oracle at the benchmark workloads' own shapes,
for a few sweeps each (the oracle runs a production sweep in tens of ms on a
host's cores):

* the small plain run: L=12, 32 samples, 2 copies, 16 temperatures in
  [0.5, 2], its whole 2048 sweeps, exchange and measurement every sweep;
* production: L=16, 1024 samples (32 words), 2 copies, 24 temperatures
  geometric in T in [0.2, 2], exchange and measurement every sweep;
* batched, uneven sizes: L=12 x 512 samples (16 T), L=14 x 384 (20 T),
  L=16 x 256 (24 T), T in [0.2, 2], as one tuned batch graph;
* large lattice: L=48, 256 samples, 2 copies, 32 temperatures in [0.5, 2]
  on the streaming engine.

Compared bit for bit: spins, integer energy / magnetisation / overlap sums
and last values, Q^2 / Q^4 moments, D histograms, every exchange mask of every
round, accepted-exchange counts, and the exp() boundary count (must be 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


SEED = 0x5EED0001


def _compare(o_gpu, o_orc, rounds):
    assert o_gpu.boundary == 0 and o_orc.boundary == 0
    assert o_gpu.n_meas == o_orc.n_meas and o_gpu.swap_rounds == o_orc.swap_rounds
    for name in ("e_sum", "e_last", "m_sum", "m_last", "q_sum", "q2_sum", "q4_sum", "hist",
                 "d_last", "swap_acc"):
        np.testing.assert_array_equal(getattr(o_gpu, name), getattr(o_orc, name), err_msg=name)
    np.testing.assert_array_equal(o_gpu.swap_log[:rounds], o_orc.swap_log[:rounds])


def _oracle(orc, L, W, T, betas, n, H=0.0):
    spins, bonds = orc.init(L, W, 2, T, SEED)
    o = orc.Observables(L, W, 2, T, log_rounds=n)
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=SEED, sweep0=0, n_sweeps=n,
            sweeps_per_swap=1, sweeps_per_meas=1, obs=o)
    return spins, o


@pytest.mark.parametrize("L,W,T,trange,n,flags", [
    (12, 1, 16, (0.5, 2.0), 2048, 0),  # the small plain run, whole length (1024 + 1024 sweeps)
    (16, 32, 24, (0.2, 2.0), 8, 0),   # production
    (48, 8, 32, (0.5, 2.0), 2, 0),    # large lattice (streaming engine)
    (48, 8, 32, (0.5, 2.0), 2, 4),    # the same, fused sweep launch (CSG_STREAM_FUSED)
])
def test_plain_engine_at_benchmark_shape(csg, orc, L, W, T, trange, n, flags):
    betas = orc.geometric_betas(T, *trange)
    with csg.Engine(L, W, 2, betas, seed=SEED, sweeps_per_swap=1, sweeps_per_meas=1,
                    flags=flags | csg.CSG_MEASURE_M, swap_log_rounds=n) as e:
        e.init_lattice()
        e.run(n)
        s_gpu, _, _ = e.get_state()
        o_gpu = e.observables()
    s_orc, o_orc = _oracle(orc, L, W, T, betas, n)
    np.testing.assert_array_equal(s_gpu, s_orc)
    _compare(o_gpu, o_orc, n)


def test_batched_mixed_workload(csg, orc):
    shapes = [(12, 16, 16), (14, 12, 20), (16, 8, 24)]  # L, words, temperatures
    n = 4
    members = [dict(L=L, n_words=W, n_copies=2, betas=orc.geometric_betas(T, 0.2, 2.0),
                    seed=SEED, sweeps_per_swap=1, sweeps_per_meas=1, flags=csg.CSG_MEASURE_M,
                    swap_log_rounds=n) for L, W, T in shapes]
    with csg.Batch(members) as b:
        for e in b.members:
            e.init_lattice()
        b.tune(8)
        b.run(n)
        got = [(e.get_state()[0], e.observables()) for e in b.members]
    for (L, W, T), m, (s_gpu, o_gpu) in zip(shapes, members, got):
        s_orc, o_orc = _oracle(orc, L, W, T, m["betas"], n)
        np.testing.assert_array_equal(s_gpu, s_orc)
        _compare(o_gpu, o_orc, n)
