"""Size-independent properties at the benchmark sizes, where the CPU oracle is
too slow to follow: the production shape (L=16, 1024 samples, 2 copies, 24
temperatures, cluster-resident kernel) and the large-lattice shape (L=48, 256
samples, 2 copies, 32 temperatures, streaming engine).

* The integer energies and overlaps that the sweep kernels accumulate with
  bit-sliced counters equal an independent recount of the final state (the
  records kernel walks every site of every lattice one sample per lane).
* A run split into several calls equals the same run in one call, bit for bit
  (spins and every accumulator).
* Exchange counts stay within the number of attempts; no exchange decision
  fell within the exp() rounding window.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


SHAPES = [
    # L, words, temperatures, T range, sweeps
    (16, 32, 24, (0.2, 2.0), 12),   # production (cluster-resident kernel)
    (48, 8, 32, (0.5, 2.0), 6),     # large lattice (streaming engine)
    (128, 1, 4, (0.5, 2.0), 2),     # the largest lattice side
    (8, 64, 16, (0.5, 2.0), 6),     # many sample words (2048 samples) at small L
]


@pytest.mark.parametrize("L,W,T,trange,n", SHAPES)
def test_counters_equal_recount_and_split_runs_agree(csg, L, W, T, trange, n):
    betas = csg.geometric_betas(T, *trange)
    N = L ** 3
    kw = dict(seed=0x5EED0001, sweeps_per_swap=1, sweeps_per_meas=1, swap_log_rounds=n)
    with csg.Engine(L, W, 2, betas, **kw) as e:
        e.init_lattice()
        e.run(n)
        s_one, _, _ = e.get_state()
        o_one = e.observables()
        rec = e.obs_records()
    with csg.Engine(L, W, 2, betas, **kw) as e:
        e.init_lattice()
        for part in (1, n // 2 - 1, n - n // 2):
            e.run(part)
        s_split, _, sweep = e.get_state()
        o_split = e.observables()
    assert sweep == n
    # split run == one run
    np.testing.assert_array_equal(s_split, s_one)
    for f in ("e_sum", "e_last", "q_sum", "q2_sum", "q4_sum", "hist", "d_last", "swap_acc",
              "swap_log"):
        np.testing.assert_array_equal(getattr(o_split, f), getattr(o_one, f), err_msg=f)
    assert o_one.n_meas == n and o_one.swap_rounds == n
    assert o_one.boundary == 0
    # counters == recount of the final state (records: e = E_bond / N, q0 = (N - 2D) / N)
    e_last = o_one.e_last  # [W][C][T][32]
    for c in range(2):
        want = (e_last[:, c].transpose(0, 2, 1).reshape(32 * W, T).astype(np.float32)
                / np.float32(N))
        np.testing.assert_array_equal(rec[:, :, c], want)
    d = o_one.d_last.transpose(0, 2, 1).reshape(32 * W, T)
    np.testing.assert_array_equal(rec[:, :, 4], (N - 2 * d).astype(np.float32) / np.float32(N))
    # the last measurement's Q sums into the histogram and the moments
    assert int(o_one.hist.sum()) == n * 32 * W * T
    assert np.all(np.abs(e_last) <= 3 * N) and np.all((0 <= o_one.d_last) & (o_one.d_last <= N))
    # exchanges: pair t is tried on rounds of its parity, each by 32 W samples per copy
    rounds = np.array([(n + 1 - (t % 2)) // 2 for t in range(T)])
    rounds[T - 1] = 0
    assert np.all(o_one.swap_acc <= rounds[None, :] * 32 * W)
    assert np.all(o_one.swap_acc[:, T - 1] == 0)
    # every logged mask sits on a pair of that round's parity
    log = o_one.swap_log[:n]  # [round][W][C][T]
    for r in range(n):
        off = [t for t in range(T) if (t % 2) != (r % 2) or t == T - 1]
        assert not log[r][:, :, off].any()
