"""Batched engine: mixed lattice sizes in one captured graph, bit-identical to
each simulation run alone (and to the oracle), autotuner leaves states intact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def members(orc):
    return [
        dict(L=8, n_words=2, n_copies=2, betas=orc.geometric_betas(8, 0.4, 2.0), seed=11,
             sweeps_per_swap=1, sweeps_per_meas=1),
        dict(L=10, n_words=1, n_copies=2, betas=orc.geometric_betas(12, 0.3, 2.0), seed=12,
             sweeps_per_swap=2, sweeps_per_meas=3),
        dict(L=12, n_words=1, n_copies=2, betas=orc.geometric_betas(16, 0.5, 2.5), seed=13,
             H=0.2, sweeps_per_swap=1, sweeps_per_meas=1),
    ]


def oracle_state(orc, m, n):
    T = len(m["betas"])
    s, b = orc.init(m["L"], m["n_words"], m["n_copies"], T, m["seed"])
    o = orc.run(s, b, L=m["L"], betas=m["betas"], H=m.get("H", 0.0), seed=m["seed"], sweep0=0,
                n_sweeps=n, sweeps_per_swap=m["sweeps_per_swap"],
                sweeps_per_meas=m["sweeps_per_meas"])
    return s, o


def test_batch_matches_oracle_and_replays(csg, orc):
    ms = members(orc)
    with csg.Batch(ms) as b:
        for e in b.members:
            e.init_lattice()
        b.run(15)
        b.run(15)  # the captured graph is replayed and continues every chain
        for m, e in zip(ms, b.members):
            s, _, sweep = e.get_state()
            o = e.observables()
            so, oo = oracle_state(orc, m, 30)
            assert sweep == 30
            np.testing.assert_array_equal(s, so)
            np.testing.assert_array_equal(o.e_sum, oo.e_sum)
            np.testing.assert_array_equal(o.q2_sum, oo.q2_sum)
            np.testing.assert_array_equal(o.hist, oo.hist)
            assert o.n_meas == oo.n_meas and o.boundary == 0


def test_sequential_equals_batched(csg, orc):
    ms = members(orc)
    states = []
    for sequential in (False, True):
        with csg.Batch(ms) as b:
            for e in b.members:
                e.init_lattice()
            (b.run_sequential if sequential else b.run)(20)
            states.append([e.get_state()[0] for e in b.members])
    for a, c in zip(*states):
        np.testing.assert_array_equal(a, c)


def test_tuner_keeps_states_and_results(csg, orc):
    ms = members(orc)
    with csg.Batch(ms) as b:
        for e in b.members:
            e.init_lattice()
        before = [e.get_state()[0] for e in b.members]
        chosen = b.tune(8)
        for m, q in zip(ms, chosen):
            G = m["n_copies"] * len(m["betas"]) // 4
            assert q >= 1 and G % q == 0
        for e, s0 in zip(b.members, before):
            np.testing.assert_array_equal(e.get_state()[0], s0)
        b.run(10)
        for m, e in zip(ms, b.members):
            np.testing.assert_array_equal(e.get_state()[0], oracle_state(orc, m, 10)[0])


def test_graph_on_caller_stream_after_state_copies(csg, orc):
    """The graph's members start in capture order through launch-completion
    edges between their first launches: launched on a fresh caller stream right
    behind csg_set_state copies, with two members of the same L (told apart by
    their state buffers) and sections longer than one launch, every member is
    still bit-equal to the oracle."""
    import torch
    ms = members(orc) + [dict(L=8, n_words=1, n_copies=2, betas=orc.geometric_betas(12, 0.5, 2.0),
                              seed=14, sweeps_per_swap=1, sweeps_per_meas=1)]
    side = torch.cuda.Stream()
    n = 1100  # two launches per member: the edges join the first ones only
    with csg.Batch(ms) as b:
        for m, e in zip(ms, b.members):
            T = len(m["betas"])
            s0, b0 = orc.init(m["L"], m["n_words"], m["n_copies"], T, m["seed"])
            e.set_state(s0, b0, 0)
        b.launch(n, side.cuda_stream)
        side.synchronize()
        for m, e in zip(ms, b.members):
            s, _, sweep = e.get_state()
            assert sweep == n
            np.testing.assert_array_equal(s, oracle_state(orc, m, n)[0])
