"""Bit-exact parity of the CUDA engine (through the C ABI) with the CPU oracle:
spins, integer energies and overlaps, every exchange decision, histograms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _compare_obs(o_gpu, o_orc, two_copies=True, with_m=False):
    assert o_gpu.n_meas == o_orc.n_meas
    assert o_gpu.swap_rounds == o_orc.swap_rounds
    assert o_gpu.boundary == 0 and o_orc.boundary == 0
    np.testing.assert_array_equal(o_gpu.e_sum, o_orc.e_sum)
    np.testing.assert_array_equal(o_gpu.e_last, o_orc.e_last)
    if with_m:
        np.testing.assert_array_equal(o_gpu.m_sum, o_orc.m_sum)
        np.testing.assert_array_equal(o_gpu.m_last, o_orc.m_last)
    np.testing.assert_array_equal(o_gpu.swap_acc, o_orc.swap_acc)
    if two_copies:
        np.testing.assert_array_equal(o_gpu.q_sum, o_orc.q_sum)
        np.testing.assert_array_equal(o_gpu.q2_sum, o_orc.q2_sum)
        np.testing.assert_array_equal(o_gpu.q4_sum, o_orc.q4_sum)
        np.testing.assert_array_equal(o_gpu.hist, o_orc.hist)
        np.testing.assert_array_equal(o_gpu.d_last, o_orc.d_last)


def test_device_init_matches_oracle(csg, orc):
    for (L, W, C_, T, seed) in [(4, 1, 2, 4, 1), (12, 2, 2, 16, 0x5EED0001), (16, 1, 1, 24, 77)]:
        betas = orc.geometric_betas(T, 0.5, 2.0)
        with csg.Engine(L, W, C_, betas, seed=seed) as e:
            e.init_lattice()
            s, b, sweep = e.get_state()
        so, bo = orc.init(L, W, C_, T, seed)
        assert sweep == 0
        np.testing.assert_array_equal(b, bo)
        np.testing.assert_array_equal(s, so)


CASES = [
    # L, W, C, T, H, sweeps, sps, spm, meas_start
    (4, 1, 2, 4, 0.0, 24, 1, 1, 0),
    (6, 2, 2, 8, 0.0, 30, 1, 2, 5),
    (8, 1, 2, 12, 0.0, 25, 3, 1, 0),
    (10, 1, 1, 8, 0.0, 20, 1, 0, 0),
    (12, 1, 2, 16, 0.0, 24, 1, 1, 0),
    (14, 1, 2, 20, 0.0, 12, 1, 1, 0),
    (16, 2, 2, 24, 0.0, 10, 1, 1, 0),
    (8, 1, 2, 8, 0.3, 20, 1, 1, 0),
    (12, 1, 2, 8, 1.7, 16, 2, 1, 0),
    (18, 1, 2, 4, 0.0, 6, 1, 1, 0),
    (24, 1, 2, 8, 0.0, 4, 1, 1, 0),
    (8, 1, 2, 64, 0.0, 8, 1, 1, 0),    # the largest ladder
    (6, 3, 1, 4, 0.2, 10, 2, 3, 1),    # the smallest ladder, one copy, H != 0
    (20, 1, 2, 12, 0.0, 5, 1, 1, 2),
]


@pytest.mark.parametrize("L,W,C_,T,H,n,sps,spm,ms", CASES)
def test_engine_matches_oracle(csg, orc, L, W, C_, T, H, n, sps, spm, ms):
    seed = 1000 + L * 7 + T
    betas = orc.geometric_betas(T, 0.4, 2.5)
    spins, bonds = orc.init(L, W, C_, T, seed)
    rounds = n // sps if sps else 0
    flags = csg.CSG_MEASURE_M
    with csg.Engine(L, W, C_, betas, H=H, seed=seed, sweeps_per_swap=sps, sweeps_per_meas=spm,
                    meas_start=ms, flags=flags, swap_log_rounds=max(rounds, 1)) as e:
        e.set_state(spins, bonds, 0)
        e.run(n // 2)
        e.run(n - n // 2)  # split: the sweep counter carries across calls
        s_gpu, b_gpu, sweep = e.get_state()
        o_gpu = e.observables()
    o_orc = orc.Observables(L, W, C_, T, log_rounds=max(rounds, 1))
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=seed, sweep0=0, n_sweeps=n,
            sweeps_per_swap=sps, sweeps_per_meas=spm, meas_start=ms, obs=o_orc)
    assert sweep == n
    np.testing.assert_array_equal(b_gpu, bonds)
    np.testing.assert_array_equal(s_gpu, spins)
    _compare_obs(o_gpu, o_orc, two_copies=(C_ == 2), with_m=True)
    if rounds:
        np.testing.assert_array_equal(o_gpu.swap_log[:rounds], o_orc.swap_log[:rounds])


@pytest.mark.parametrize("qc", [1, 2, 6])
def test_plan_variants_agree(csg, orc, qc):
    """Every split of the quads over a cluster gives the same bits."""
    L, W, C_, T, n = 8, 1, 2, 24, 12
    betas = orc.geometric_betas(T, 0.3, 2.0)
    spins, bonds = orc.init(L, W, C_, T, 5)
    csg.set_plan_override(qc)
    try:
        with csg.Engine(L, W, C_, betas, seed=5, sweeps_per_swap=1, sweeps_per_meas=1) as e:
            e.set_state(spins, bonds, 0)
            e.run(n)
            s_gpu, _, _ = e.get_state()
            o_gpu = e.observables()
    finally:
        csg.set_plan_override(None)
    o_orc = orc.run(spins, bonds, L=L, betas=betas, H=0.0, seed=5, sweep0=0, n_sweeps=n,
                    sweeps_per_swap=1, sweeps_per_meas=1)
    np.testing.assert_array_equal(s_gpu, spins)
    _compare_obs(o_gpu, o_orc)


# (L, T, quads per CTA, threads per quad): both column splits of each L, and
# teams that are not whole warps (L = 6, 10, 12, 14), so that warps hold
# lanes of two quads and padding threads
TILES = [
    (6, 8, 1, 36), (6, 8, 4, 36),
    (8, 8, 4, 32), (8, 8, 2, 64),
    (10, 8, 1, 50), (10, 8, 4, 100), (10, 8, 2, 50),
    (12, 16, 4, 72), (12, 16, 2, 144), (12, 16, 1, 72),
    (14, 20, 5, 98), (14, 20, 2, 98), (14, 20, 2, 196),
    (16, 24, 3, 128), (16, 24, 2, 256), (16, 24, 1, 128),
]


@pytest.mark.parametrize("L,T,qc,tpq", TILES)
@pytest.mark.parametrize("H", [0.0, 0.4])
def test_tile_variants_match_oracle(csg, orc, L, T, qc, tpq, H):
    """Every tile (quads per CTA x threads per quad) gives the oracle's bits,
    with exchange and measurement every sweep, at H = 0 and H != 0."""
    W, C_, n = 1, 2, 6
    seed = 4242 + L
    betas = orc.geometric_betas(T, 0.3, 2.0)
    spins, bonds = orc.init(L, W, C_, T, seed)
    csg.set_plan_override(qc, tpq)
    if H != 0 and tpq == L * L // 2 and (qc * tpq + 31) // 32 * 32 > 384:
        # the general-field kernel walking whole columns takes at most 384
        # threads per CTA (168 registers each): the tile is refused, not run
        try:
            with pytest.raises(csg.CsgError, match="plan override exceeds device limits"):
                csg.query_plan(L, W, C_, betas, H=H)
        finally:
            csg.set_plan_override(None)
        return
    try:
        plan = csg.query_plan(L, W, C_, betas, H=H)
        assert (plan.quads_per_cta, plan.threads_per_quad) == (qc, tpq)
        with csg.Engine(L, W, C_, betas, H=H, seed=seed, sweeps_per_swap=1, sweeps_per_meas=1,
                        flags=csg.CSG_MEASURE_M, swap_log_rounds=n) as e:
            e.set_state(spins, bonds, 0)
            e.run(n)
            s_gpu, _, _ = e.get_state()
            o_gpu = e.observables()
    finally:
        csg.set_plan_override(None)
    o_orc = orc.Observables(L, W, C_, T, log_rounds=n)
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=seed, sweep0=0, n_sweeps=n,
            sweeps_per_swap=1, sweeps_per_meas=1, obs=o_orc)
    np.testing.assert_array_equal(s_gpu, spins)
    _compare_obs(o_gpu, o_orc, with_m=True)
    np.testing.assert_array_equal(o_gpu.swap_log[:n], o_orc.swap_log[:n])


def test_long_run_crosses_launch_boundary(csg, orc):
    """More sweeps than one launch holds; resumes mid-schedule."""
    L, W, C_, T = 4, 1, 2, 8
    betas = orc.geometric_betas(T, 0.5, 2.0)
    spins, bonds = orc.init(L, W, C_, T, 9)
    n = 1500
    with csg.Engine(L, W, C_, betas, seed=9, sweeps_per_swap=2, sweeps_per_meas=3,
                    meas_start=700) as e:
        e.set_state(spins, bonds, 123)
        e.run(n)
        s_gpu, _, sweep = e.get_state()
        o_gpu = e.observables()
    o_orc = orc.run(spins, bonds, L=L, betas=betas, H=0.0, seed=9, sweep0=123, n_sweeps=n,
                    sweeps_per_swap=2, sweeps_per_meas=3, meas_start=700)
    assert sweep == 123 + n
    np.testing.assert_array_equal(s_gpu, spins)
    _compare_obs(o_gpu, o_orc)


def test_obs_records_and_checkpoint_round_trip(csg, orc):
    L, W, T, H = 8, 2, 24, 0.1875
    betas = csg.reference_betas(T)
    spins, bonds = orc.init(L, W, 2, T, 31)
    with csg.Engine(L, W, 2, betas, H=H, seed=31, sweeps_per_swap=16) as e:
        e.set_state(spins, bonds, 0)
        e.run(40)
        s_gpu, _, _ = e.get_state()
        rec = e.obs_records()
        ref = e.save_checkpoint()
        e.load_checkpoint(ref, sweep=40)
        s2, b2, sweep = e.get_state()
    orc.run(spins, bonds, L=L, betas=betas, H=H, seed=31, sweep0=0, n_sweeps=40,
            sweeps_per_swap=16)
    np.testing.assert_array_equal(s_gpu, spins)
    np.testing.assert_array_equal(rec, orc.obs_records(spins, bonds, L, H))
    np.testing.assert_array_equal(ref, orc.to_ref_lattice(spins, bonds, L))
    np.testing.assert_array_equal(s2, spins)
    np.testing.assert_array_equal(b2, bonds)
    assert sweep == 40


def test_corrupt_checkpoint_is_rejected(csg, orc):
    L, T = 6, 8
    betas = orc.geometric_betas(T, 0.5, 2.0)
    spins, bonds = orc.init(L, 1, 2, T, 3)
    ref = orc.to_ref_lattice(spins, bonds, L)
    ref[2, 5] ^= 1 << 26  # one end of a bond flipped
    with csg.Engine(L, 1, 2, betas, seed=3) as e:
        with pytest.raises(csg.CsgError, match="bond"):
            e.load_checkpoint(ref)
        with pytest.raises(csg.CsgError, match="size"):
            e.load_checkpoint(ref[:-1])


def test_device_entry_point_on_torch_memory(csg, orc):
    """csg_pt_run_device on caller-owned device buffers (no engine)."""
    import torch
    L, W, C_, T, n = 12, 2, 2, 16, 10
    betas = orc.geometric_betas(T, 0.5, 2.0)
    spins, bonds = orc.init(L, W, C_, T, 21)
    cfg, _keep = csg.make_config(L, W, C_, betas, seed=21, sweeps_per_swap=1, sweeps_per_meas=1)
    ds = torch.from_numpy(spins.view(np.int32)).cuda()
    db = torch.from_numpy(bonds.view(np.int32)).cuda()
    e_sum = torch.zeros((W, C_, T, 32), dtype=torch.int64, device="cuda")
    q2 = torch.zeros((W, T, 32), dtype=torch.int64, device="cuda")
    bnd = torch.zeros(1, dtype=torch.int64, device="cuda")
    obs = csg.DeviceObs(e_sum=e_sum.data_ptr(), q2_sum=q2.data_ptr(), boundary=bnd.data_ptr())
    csg.run_device(cfg, ds.data_ptr(), db.data_ptr(), obs, 0, n,
                   torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    o = orc.run(spins, bonds, L=L, betas=betas, H=0.0, seed=21, sweep0=0, n_sweeps=n,
                sweeps_per_swap=1, sweeps_per_meas=1)
    np.testing.assert_array_equal(ds.cpu().numpy().view(np.uint32), spins)
    np.testing.assert_array_equal(e_sum.cpu().numpy(), o.e_sum)
    np.testing.assert_array_equal(q2.cpu().numpy(), o.q2_sum)
    assert int(bnd.item()) == 0


def test_plan_query(csg):
    p = csg.query_plan(16, 32, 2, csg.geometric_betas(24, 0.2, 2.0))
    assert p.quads_per_cta * p.ctas_per_word == 12
    assert p.smem_bytes <= 227 * 1024
