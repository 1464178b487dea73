"""The streaming engine (lattices whose temperature quads do not fit in a
cluster's shared memory, L > 24, or any L with CSG_ENGINE_STREAM): bit-exact
parity with the CPU oracle and with the cluster-resident kernel."""
import numpy as np
import pytest


def test_large_lattice_plan_and_footprint(csg):
    betas = np.linspace(2.0, 0.5, 8)
    # colour launches by default
    p = csg.query_plan(32, 2, 2, betas)
    assert (p.quads_per_cta, p.ctas_per_word, p.threads_per_quad, p.smem_bytes) == (0, 0, 256, 0)
    # the fused sweep launch (L <= 58) when asked for: one CTA of L*L/2 /
    # sites-per-thread threads per quad, a ring of 2 x 4 half z-planes (L*L/2 x
    # 16 bytes each)
    F = csg.CSG_STREAM_FUSED
    p = csg.query_plan(32, 2, 2, betas, flags=F)
    assert (p.quads_per_cta, p.ctas_per_word, p.threads_per_quad, p.smem_bytes) == \
        (1, 4, 512, 8 * 512 * 16)
    p = csg.query_plan(48, 1, 2, betas, flags=F)
    assert (p.threads_per_quad, p.smem_bytes) == (384, 8 * 1152 * 16)
    p = csg.query_plan(58, 1, 2, betas, flags=F)
    assert (p.threads_per_quad, p.smem_bytes) == (448, 8 * 1682 * 16)
    # colour launches beyond it
    p = csg.query_plan(60, 1, 2, betas, flags=F)
    assert (p.quads_per_cta, p.ctas_per_word, p.threads_per_quad, p.smem_bytes) == (0, 0, 256, 0)
    N = 32 ** 3
    spins = 2 * 2 * 8 * N * 4
    assert csg.footprint(32, 2, 2, betas) > spins + 2 * 3 * N * 4
    # the forced streaming engine plans the same way at small L
    p = csg.query_plan(8, 1, 2, betas, flags=csg.CSG_ENGINE_STREAM)
    assert (p.quads_per_cta, p.threads_per_quad) == (0, 256)
    p = csg.query_plan(8, 1, 2, betas, flags=csg.CSG_ENGINE_STREAM | F)
    assert (p.quads_per_cta, p.threads_per_quad, p.smem_bytes) == (1, 32, 8 * 32 * 16)
    assert csg.footprint(8, 1, 2, betas, flags=csg.CSG_ENGINE_STREAM) > \
        csg.footprint(8, 1, 2, betas)


@pytest.mark.parametrize("L", [25, 130, 2])
def test_large_lattice_limits(csg, L):
    with pytest.raises(csg.CsgError):
        csg.query_plan(L, 1, 2, np.linspace(2.0, 0.5, 8))


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _compare(o_gpu, o_orc, two_copies):
    assert o_gpu.n_meas == o_orc.n_meas
    assert o_gpu.swap_rounds == o_orc.swap_rounds
    assert o_gpu.boundary == 0 and o_orc.boundary == 0
    for f in ("e_sum", "e_last", "m_sum", "m_last", "swap_acc"):
        np.testing.assert_array_equal(getattr(o_gpu, f), getattr(o_orc, f), err_msg=f)
    if two_copies:
        for f in ("q_sum", "q2_sum", "q4_sum", "hist", "d_last"):
            np.testing.assert_array_equal(getattr(o_gpu, f), getattr(o_orc, f), err_msg=f)


STREAM_CASES = [
    # L, W, C, T, H, sweeps, sps, spm, meas_start, forced
    (26, 1, 2, 12, 0.0, 6, 1, 1, 0, False),
    (28, 2, 2, 8, 0.0, 5, 1, 2, 1, False),
    (32, 1, 2, 16, 0.0, 4, 1, 1, 0, False),
    (32, 1, 1, 8, 0.0, 4, 2, 1, 0, False),
    (30, 1, 2, 8, 0.7, 5, 1, 1, 0, False),
    (48, 1, 2, 4, 0.0, 3, 1, 1, 0, False),
    (64, 1, 2, 4, 0.0, 2, 1, 1, 0, False),
    (8, 2, 2, 12, 0.0, 20, 1, 1, 0, True),
    (12, 1, 2, 8, 1.3, 16, 2, 1, 3, True),
    (16, 1, 1, 24, 0.0, 10, 3, 2, 0, True),
    (26, 1, 2, 64, 0.0, 3, 1, 1, 0, False),   # the largest ladder
    (34, 1, 2, 4, 1.1, 3, 1, 1, 0, False),
    (4, 1, 2, 8, 0.0, 12, 1, 1, 0, True),     # the smallest lattice
]

# The fused sweep launch (CSG_STREAM_FUSED): its edges (the smallest lattice,
# one warp per CTA; the largest; three and four sites per thread), the general
# field, magnetisations, sparse schedules and one copy.
FUSED_CASES = [
    (26, 1, 2, 12, 0.0, 6, 1, 1, 0, False),
    (32, 1, 1, 8, 0.0, 4, 2, 1, 0, False),
    (30, 1, 2, 8, 0.7, 5, 1, 1, 0, False),
    (48, 1, 2, 4, 0.0, 3, 1, 1, 0, False),
    (58, 1, 2, 4, 0.0, 2, 1, 1, 0, False),    # the largest lattice of the fused sweep launch
    (60, 1, 1, 4, 0.0, 2, 1, 1, 0, False),    # beyond it: colour launches
    (40, 1, 2, 8, 0.9, 3, 1, 1, 0, False),    # general field, two sites per thread
    (8, 2, 2, 12, 0.0, 20, 1, 1, 0, True),
    (4, 1, 2, 8, 0.0, 12, 1, 1, 0, True),     # the smallest lattice: a CTA of one warp
    (12, 1, 2, 8, 1.3, 16, 2, 1, 3, True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("L,W,C_,T,H,n,sps,spm,ms,forced", STREAM_CASES)
def test_stream_engine_matches_oracle(csg, orc, L, W, C_, T, H, n, sps, spm, ms, forced):
    _check_stream_case(csg, orc, L, W, C_, T, H, n, sps, spm, ms, forced, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("L,W,C_,T,H,n,sps,spm,ms,forced", FUSED_CASES)
def test_stream_fused_matches_oracle(csg, orc, L, W, C_, T, H, n, sps, spm, ms, forced):
    _check_stream_case(csg, orc, L, W, C_, T, H, n, sps, spm, ms, forced, csg.CSG_STREAM_FUSED)


def _check_stream_case(csg, orc, L, W, C_, T, H, n, sps, spm, ms, forced, extra_flags):
    _gpu()
    seed = 2000 + L * 5 + T
    betas = orc.geometric_betas(T, 0.4, 2.5)
    spins, bonds = orc.init(L, W, C_, T, seed)
    rounds = n // sps if sps else 0
    flags = csg.CSG_MEASURE_M | (csg.CSG_ENGINE_STREAM if forced else 0) | extra_flags
    with csg.Engine(L, W, C_, betas, H=H, seed=seed, sweeps_per_swap=sps, sweeps_per_meas=spm,
                    meas_start=ms, flags=flags, swap_log_rounds=max(rounds, 1)) as e:
        e.set_state(spins, bonds, 0)
        e.run(n // 2)
        e.run(n - n // 2)
        s_gpu, b_gpu, sweep = e.get_state()
        o_gpu = e.observables()
    o_orc = orc.Observables(L, W, C_, T, log_rounds=max(rounds, 1))
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=seed, sweep0=0, n_sweeps=n,
            sweeps_per_swap=sps, sweeps_per_meas=spm, meas_start=ms, obs=o_orc)
    assert sweep == n
    np.testing.assert_array_equal(b_gpu, bonds)
    np.testing.assert_array_equal(s_gpu, spins)
    _compare(o_gpu, o_orc, C_ == 2)
    if rounds:
        np.testing.assert_array_equal(o_gpu.swap_log[:rounds], o_orc.swap_log[:rounds])


@pytest.mark.gpu
def test_stream_equals_resident_production_shape(csg, orc):
    """Both engines give the same bits on a production-shaped state (L=16,
    2 words, 2 copies, 24 temperatures, exchange and measurement every sweep)."""
    _gpu()
    L, W, C_, T, n = 16, 2, 2, 24, 64
    betas = orc.geometric_betas(T, 0.5, 5.0)
    out = []
    for flags in (0, csg.CSG_ENGINE_STREAM):
        with csg.Engine(L, W, C_, betas, seed=0x5EED0001, word0=3, sweeps_per_swap=1,
                        sweeps_per_meas=1, flags=flags) as e:
            e.init_lattice()
            e.run(n)
            s, _, _ = e.get_state()
            out.append((s, e.observables()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    _compare(out[0][1], out[1][1], True)


@pytest.mark.gpu
def test_large_lattice_records_and_checkpoint(csg, orc):
    """Observable records and the reference checkpoint format at L=32."""
    _gpu()
    L, W, C_, T, seed = 32, 1, 2, 8, 31
    betas = orc.geometric_betas(T, 0.5, 2.0)
    with csg.Engine(L, W, C_, betas, seed=seed, sweeps_per_swap=1) as e:
        e.init_lattice()
        e.run(3)
        s, b, _ = e.get_state()
        rec = e.obs_records()
        ref = e.save_checkpoint()
    np.testing.assert_array_equal(rec, orc.obs_records(s, b, L=L, H=0.0))
    np.testing.assert_array_equal(ref, orc.to_ref_lattice(s, b, L))
    with csg.Engine(L, W, C_, betas, seed=seed, sweeps_per_swap=1) as e2:
        e2.set_state(np.zeros_like(s), b, 0)
        e2.load_checkpoint(ref, sweep=3)
        s2, _, sweep = e2.get_state()
    assert sweep == 3
    np.testing.assert_array_equal(s2, s)


@pytest.mark.gpu
def test_batch_rejects_streaming_members(csg):
    _gpu()
    betas = np.linspace(2.0, 0.5, 8)
    with pytest.raises(csg.CsgError, match="cluster-resident"):
        csg.Batch([dict(L=32, n_words=1, n_copies=2, betas=betas)])
