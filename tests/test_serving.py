"""Serving with continuous batching: requests of different L, sample counts and
ladders admitted against a memory budget while others run; each result equals
the same request run alone, bit for bit."""
import time

import numpy as np
import pytest


def request(i):
    L = [8, 10, 12, 14, 16, 8][i % 6]
    T = [8, 12, 16, 8, 12, 20][i % 6]
    return dict(L=L, n_words=1 + i % 2, n_copies=2,
                betas=1.0 / (0.3 * (2.0 / 0.3) ** (np.arange(T) / (T - 1))), seed=1000 + i,
                sweeps_per_swap=1, sweeps_per_meas=2), 40 + 12 * i


def test_footprint_and_validation(csg):
    kw, _ = request(0)
    fp = csg.footprint(**kw)
    N = kw["L"] ** 3
    assert fp > kw["n_words"] * 2 * len(kw["betas"]) * N * 4  # at least the spins
    srv = csg.Server(fp * 3, max_active=4, sweeps_per_launch=16)
    with pytest.raises(csg.CsgError):
        srv.submit(10, **dict(kw, n_copies=3))
    with pytest.raises(csg.CsgError, match="budget"):
        big = dict(kw, n_words=64, L=24)
        srv.submit(10, **big)
    srv.close()


@pytest.mark.gpu
def test_mixed_requests_equal_alone(csg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    reqs = [request(i) for i in range(6)]
    budget = 3 * max(csg.footprint(**kw) for kw, _ in reqs)  # forces queueing
    results, peak_active = {}, 0
    with csg.Server(budget, max_active=8, sweeps_per_launch=16) as srv:
        ids = {}
        for k, (kw, n) in enumerate(reqs):
            ids[srv.submit(n, **kw)] = k
            if k % 2 == 1:  # arrivals while earlier requests run
                done, na, nq = srv.poll()
                peak_active = max(peak_active, na)
                for d in done:
                    results[ids[d]] = srv.result(d, with_spins=True)
        deadline = time.time() + 120
        while len(results) < len(reqs) and time.time() < deadline:
            done, na, nq = srv.poll()
            peak_active = max(peak_active, na)
            for d in done:
                results[ids[d]] = srv.result(d, with_spins=True)
            time.sleep(0.001)
    assert len(results) == len(reqs)
    # never more active requests than the smallest footprints that fit the budget
    fps = sorted(csg.footprint(**kw) for kw, _ in reqs)
    fit = max(k for k in range(len(fps) + 1) if sum(fps[:k]) <= budget)
    assert 1 < peak_active <= fit < len(reqs)
    for k, (kw, n) in enumerate(reqs):
        with csg.Engine(**kw) as e:
            e.init_lattice()
            e.run(n)
            s, _, _ = e.get_state()
            o = e.observables()
        o_srv, s_srv = results[k]
        np.testing.assert_array_equal(s_srv, s)
        np.testing.assert_array_equal(o_srv.e_sum, o.e_sum)
        np.testing.assert_array_equal(o_srv.q2_sum, o.q2_sum)
        assert o_srv.n_meas == o.n_meas


@pytest.mark.gpu
def test_request_that_cannot_be_allocated_completes_with_an_error(csg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    small, n = request(0)
    # L=128, 8192 samples, 2 copies, 64 temperatures: 275 GB of spins, more
    # than the device holds, inside a 1 TiB budget
    huge = dict(L=128, n_words=256, n_copies=2, betas=np.linspace(0.5, 2.0, 64), seed=7)
    assert csg.footprint(**huge) > 200e9
    with csg.Server(1 << 40, max_active=4, sweeps_per_launch=16) as srv:
        a = srv.submit(n, **small)
        b = srv.submit(10, **huge)
        c = srv.submit(n, **dict(small, seed=2000))
        done, deadline = set(), time.time() + 60
        while len(done) < 3 and time.time() < deadline:
            done.update(srv.poll()[0])
            time.sleep(0.001)
        assert done == {a, b, c}
        with pytest.raises(csg.CsgError, match="cudaMalloc"):
            srv.result(b)
        o_a, o_c = srv.result(a), srv.result(c)
        assert srv.poll()[1:] == (0, 0)
    with csg.Engine(**small) as e:
        e.init_lattice()
        e.run(n)
        o = e.observables()
    np.testing.assert_array_equal(o_a.e_sum, o.e_sum)
    assert o_c.n_meas == o.n_meas


def test_request_without_a_device_completes_with_an_error(csg):
    """Host-side failure path: with no CUDA device the engine of an admitted
    request cannot be created; the request is reported completed and its
    result call raises the creation error (no GPU involved)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("needs a host without a CUDA device")
    kw, n = request(0)
    with csg.Server(1 << 30, max_active=2, sweeps_per_launch=16) as srv:
        a = srv.submit(n, **kw)
        b = srv.submit(n, **dict(kw, seed=5))
        done, na, nq = srv.poll()
        assert sorted(done) == [a, b] and (na, nq) == (0, 0)
        for r in (a, b):
            with pytest.raises(csg.CsgError, match=f"request {r}"):
                srv.result(r)
        with pytest.raises(csg.CsgError, match="unknown request"):
            srv.result(a)
