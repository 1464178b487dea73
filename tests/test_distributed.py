"""Sample sharding over ranks (spin-glass_b200/distributed.py).

On CPU: two gloo ranks run their shards on an oracle-backed stand-in engine
and gather to rank 0; the result must equal the unsplit run bit for bit.  A
rank that fails before the gather makes the other rank fail too (no hang).
On the GPU: shards with word0 offsets equal the unsplit engine."""
import os
import pathlib
import socket
import sys
import time

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
L, W, C, T, SEED, N_SWEEPS = 6, 3, 2, 8, 77, 6


def _betas():
    return 1.0 / (0.5 * (4.0 ** (np.arange(T) / (T - 1))))


class OracleEngine:
    """Stand-in with the Engine methods ShardedEngine uses, computed by the oracle."""

    def __init__(self, L_, n_words, n_copies, betas, word0=0, seed=1, **kw):
        from oracle import oracle as orc
        self.orc, self.L, self.W, self.C = orc, L_, n_words, n_copies
        self.betas, self.word0, self.seed, self.kw = np.asarray(betas), word0, seed, kw
        self.obs = orc.Observables(L_, n_words, n_copies, len(betas))
        self.sweep = 0

    def init_lattice(self):
        self.spins, self.bonds = self.orc.init(self.L, self.W, self.C, len(self.betas), self.seed,
                                               self.word0)

    def run(self, n):
        self.orc.run(self.spins, self.bonds, L=self.L, betas=self.betas, H=0.0, seed=self.seed,
                     sweep0=self.sweep, n_sweeps=n, obs=self.obs, word0=self.word0, **self.kw)
        self.sweep += n

    def observables(self):
        return self.obs


def _load_package():
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT))
    from conftest import load_package
    return load_package()


def _worker(rank, world, port, out_dir, fail_rank):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        if rank == fail_rank:
            raise RuntimeError(f"rank {rank} fails before the gather")
        csg = _load_package()
        import importlib
        distributed = importlib.import_module("spin_glass_b200.distributed")
        sh = distributed.ShardedEngine(L, W, C, _betas(), engine_factory=OracleEngine, seed=SEED,
                                       sweeps_per_swap=1, sweeps_per_meas=1)
        sh.init_lattice()
        sh.run(N_SWEEPS)
        g = sh.gather_observables()
        if rank == 0:
            np.savez(pathlib.Path(out_dir) / "gathered.npz", **{k: np.asarray(v) for k, v in g.items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges():
    sys.path.insert(0, str(ROOT / "spin-glass_b200"))
    from distributed import shard
    assert [shard(10, 4, r) for r in range(4)] == [(0, 3), (3, 3), (6, 2), (8, 2)]
    assert sum(shard(7, 3, r)[1] for r in range(3)) == 7
    with pytest.raises(ValueError):
        shard(1, 2, 0)


def test_two_gloo_ranks_equal_unsplit_run(orc, tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), -1), nprocs=2, join=True)
    g = np.load(tmp_path / "gathered.npz")
    s, b = orc.init(L, W, C, T, SEED)
    o = orc.run(s, b, L=L, betas=_betas(), H=0.0, seed=SEED, sweep0=0, n_sweeps=N_SWEEPS,
                sweeps_per_swap=1, sweeps_per_meas=1)
    for f in ("e_sum", "q_sum", "q2_sum", "q4_sum", "e_last", "d_last", "hist", "swap_acc"):
        np.testing.assert_array_equal(g[f], getattr(o, f), err_msg=f)
    assert int(g["n_meas"]) == o.n_meas == N_SWEEPS and int(g["boundary"]) == 0


def test_failing_rank_does_not_hang_the_other(tmp_path):
    import torch.multiprocessing as mp
    ctx = mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), 1), nprocs=2, join=False)
    deadline = time.time() + 90
    failed = False
    try:
        while time.time() < deadline:
            try:
                if ctx.join(timeout=1):
                    break
            except Exception:
                failed = True
                break
    finally:
        for p in ctx.processes:
            if p.is_alive():
                p.kill()
    assert failed, "the failing rank must surface as an error"
    for p in ctx.processes:
        p.join(timeout=30)
        assert not p.is_alive()
    assert not (tmp_path / "gathered.npz").exists()


@pytest.mark.gpu
def test_word_shards_equal_unsplit_engine(csg, orc):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    betas, Lg, Wg = _betas(), 8, 3
    kw = dict(seed=SEED, sweeps_per_swap=1, sweeps_per_meas=1)
    with csg.Engine(Lg, Wg, C, betas, **kw) as e:
        e.init_lattice()
        e.run(12)
        s_all = e.get_state()[0]
        o_all = e.observables()
    parts = []
    for first, n in [(0, 1), (1, 2)]:
        with csg.Engine(Lg, n, C, betas, word0=first, **kw) as e:
            e.init_lattice()
            e.run(12)
            parts.append((e.get_state()[0], e.observables()))
    np.testing.assert_array_equal(np.concatenate([p[0] for p in parts]), s_all)
    np.testing.assert_array_equal(np.concatenate([p[1].e_sum for p in parts]), o_all.e_sum)
    np.testing.assert_array_equal(parts[0][1].hist + parts[1][1].hist, o_all.hist)
