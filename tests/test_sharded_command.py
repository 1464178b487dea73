"""The sharded `csg <sim_dir> <H>` command (spin-glass_b200/csg_sharded.py).

Two gloo ranks on CPU run the command with an oracle-backed stand-in for the
per-rank engine.  What must hold (as for the single-GPU command,
tests/test_cli.py):

* <H>-obs.bin and <H>-chkpt.bin equal the unsplit chain's records and
  reference checkpoint (oracle), and the sidecar holds the sweep count and
  seed;
* a run split over two invocations writes the same bytes as one run;
* without a seed in csg.conf every rank uses rank 0's start time;
* configuration errors, and an error on one rank only, end every rank with
  exit code 1 (no rank waits in a collective), and the log keeps the message.
"""
import json
import pathlib
import socket
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
L, NDIS, NREP, SBSHFL, SBMEAS, SEED, H = 6, 96, 8, 1, 4, 4242, "0.25"


class OracleEngine:
    """Stand-in with the Engine methods the command uses, computed by the oracle."""

    def __init__(self, L_, n_words, n_copies, betas, word0=0, seed=1, H=0.0, flags=0,
                 sweeps_per_swap=1, sweeps_per_meas=0, fail_at=None):
        from oracle import oracle as orc
        self.orc, self.L, self.W, self.C = orc, L_, n_words, n_copies
        self.T = len(betas)
        self.betas, self.word0, self.seed, self.H = np.asarray(betas), word0, seed, H
        self.sps, self.spm, self.fail_at = sweeps_per_swap, sweeps_per_meas, fail_at
        self.sweep, self.n_rec = 0, 0

    def init_lattice(self):
        self.spins, self.bonds = self.orc.init(self.L, self.W, self.C, self.T, self.seed,
                                               self.word0)

    def run(self, n):
        self.orc.run(self.spins, self.bonds, L=self.L, betas=self.betas, H=self.H, seed=self.seed,
                     sweep0=self.sweep, n_sweeps=n, sweeps_per_swap=self.sps,
                     sweeps_per_meas=self.spm, word0=self.word0)
        self.sweep += n

    def obs_records(self):
        self.n_rec += 1
        if self.fail_at is not None and self.n_rec == self.fail_at:
            raise RuntimeError("device lost (planted)")
        return self.orc.obs_records(self.spins, self.bonds, self.L, self.H)

    def save_checkpoint(self):
        return self.orc.to_ref_lattice(self.spins, self.bonds, self.L)

    def load_checkpoint(self, ref, sweep=0):
        assert ref.shape == (64 * self.W, self.L ** 3)
        self.spins, self.bonds = self.orc.from_ref_lattice(ref, self.L, self.T)
        self.sweep = sweep


def _load_package():
    sys.path.insert(0, str(ROOT / "tests"))
    sys.path.insert(0, str(ROOT))
    from conftest import load_package
    return load_package()


def _worker(rank, world, port, jobs, out_dir):
    """Runs each job (sim_dir, H, log_dir, failing rank, failing record call)
    as one invocation of the command on this rank; saves the exit codes."""
    import datetime
    import importlib
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        _load_package()
        cmd = importlib.import_module("spin_glass_b200.csg_sharded")
        codes = []
        for sim_dir, h, log_dir, fail_rank, fail_at in jobs:
            def factory(*a, **kw):
                return OracleEngine(*a, fail_at=fail_at if rank == fail_rank else None, **kw)
            codes.append(cmd.run(sim_dir, h, engine_factory=factory, log_dir=log_dir))
        (pathlib.Path(out_dir) / f"rc-{rank}.json").write_text(json.dumps(codes))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(jobs, out_dir, world=2):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), jobs, str(out_dir)), nprocs=world, join=True)
    return [json.loads((out_dir / f"rc-{r}.json").read_text()) for r in range(world)]


def _conf(d: pathlib.Path, **kv):
    d.mkdir(parents=True, exist_ok=True)
    (d / "csg.conf").write_text("".join(f"{k} = {v}\n" for k, v in kv.items()))
    return str(d)


def _expected(orc, seed, n_sections):
    """Records of every section and the final reference checkpoint of the
    unsplit chain, computed by the oracle (the ladder as csg_main.cpp makes it)."""
    ratio = (0.5 / 2.0) ** (1.0 / (NREP - 1))
    betas = np.array([np.float32(ratio ** r * 2.0) for r in range(NREP)], np.float64)
    spins, bonds = orc.init(L, NDIS // 32, 2, NREP, seed)
    recs = []
    for sec in range(n_sections):
        orc.run(spins, bonds, L=L, betas=betas, H=float(H), seed=seed, sweep0=SBMEAS * sec,
                n_sweeps=SBMEAS, sweeps_per_swap=SBSHFL, sweeps_per_meas=SBMEAS)
        recs.append(orc.obs_records(spins, bonds, L, float(H)))
    return np.stack(recs), orc.to_ref_lattice(spins, bonds, L)


def test_ladder_and_parsing_match_the_single_gpu_command(csg):
    cmd = __import__("importlib").import_module("spin_glass_b200.csg_sharded")
    # eamsim.cu:728-737 with beta_max 2, beta_min 0.125, 24 temperatures
    np.testing.assert_array_equal(cmd.ladder(24, 2.0, 0.125), csg.reference_betas(24))
    assert cmd._stoi(" 12abc") == 12 and cmd._stoull_auto("0x1F") == 31
    assert cmd._stoull_auto("017") == 15 and cmd._stoull_auto("-1") == 2 ** 64 - 1
    assert cmd.parse_field("0.25") == 0.25 and cmd.parse_field("1e-1") == float(np.float32(0.1))
    with pytest.raises(cmd.Failure):
        cmd.parse_field("x")


def test_sharded_command_equals_the_unsplit_chain(orc, tmp_path):
    small = dict(L=L, NDIS=NDIS, NREP=NREP, SBSHFL=SBSHFL, SBMEAS=SBMEAS, beta_max=2.0,
                 beta_min=0.5)
    one = _conf(tmp_path / "one", SPFILE=2 * SBMEAS, seed=SEED, **small)
    split = _conf(tmp_path / "split", SPFILE=SBMEAS, seed=SEED, **small)
    fresh = _conf(tmp_path / "fresh", SPFILE=SBMEAS, **small)
    logs = tmp_path / "logs"
    logs.mkdir()
    jobs = [(one, H, str(logs), -1, None), (split, H, str(logs), -1, None),
            (split, H, str(logs), -1, None), (fresh, H, str(logs), -1, None)]
    assert _spawn(jobs, tmp_path) == [[0, 0, 0, 0]] * 2
    assert not list(logs.glob("*.log")), "the log is removed on success"
    recs, chk = _expected(orc, SEED, 2)
    files = {}
    for d in (one, split):
        p = pathlib.Path(d)
        obs = np.fromfile(p / "0.2500-obs.bin", np.float32)
        np.testing.assert_array_equal(obs.reshape(recs.shape), recs)
        ref = np.fromfile(p / "0.2500-chkpt.bin", np.uint32)
        np.testing.assert_array_equal(ref.reshape(chk.shape), chk)
        assert (p / "0.2500-chkpt.csg").read_text().split() == ["csg-resume-v1", "8", str(SEED)]
        files[d] = [(p / f).read_bytes() for f in ("0.2500-obs.bin", "0.2500-chkpt.bin")]
    assert files[one] == files[split]
    # no seed in csg.conf: every rank took rank 0's start time as the seed
    side = (pathlib.Path(fresh) / "0.2500-chkpt.csg").read_text().split()
    assert side[:2] == ["csg-resume-v1", "4"]
    recs_f, chk_f = _expected(orc, int(side[2]), 1)
    obs = np.fromfile(pathlib.Path(fresh) / "0.2500-obs.bin", np.float32)
    np.testing.assert_array_equal(obs.reshape(recs_f.shape), recs_f)
    ref = np.fromfile(pathlib.Path(fresh) / "0.2500-chkpt.bin", np.uint32)
    np.testing.assert_array_equal(ref.reshape(chk_f.shape), chk_f)


def test_errors_end_every_rank(tmp_path):
    small = dict(L=L, NREP=NREP, SBSHFL=SBSHFL, SBMEAS=SBMEAS, SPFILE=2 * SBMEAS, seed=SEED)
    one_word = _conf(tmp_path / "one_word", NDIS=32, **small)       # 1 word for 2 ranks
    bad_key = _conf(tmp_path / "bad_key", NDIS=NDIS, colour=1, **small)
    lost = _conf(tmp_path / "lost", NDIS=NDIS, **small)             # rank 1 fails mid-run
    jobs = []
    for name, d, h, fail_at in [("one_word", one_word, H, None), ("bad_key", bad_key, H, None),
                                ("range", one_word, "4.5", None), ("lost", lost, H, 2)]:
        (tmp_path / name / "logs").mkdir(parents=True, exist_ok=True)
        jobs.append((d, h, str(tmp_path / name / "logs"), 1, fail_at))
    assert _spawn(jobs, tmp_path) == [[1, 1, 1, 1]] * 2
    msgs = {}
    for name in ("one_word", "bad_key", "range", "lost"):
        kept = list((tmp_path / name / "logs").glob("*.log"))
        assert len(kept) == 1, name  # the log is kept on failure (main.cu:70-75)
        msgs[name] = kept[0].read_text()
    assert "need at least one word per rank" in msgs["one_word"]
    assert "unknown key in csg.conf: colour" in msgs["bad_key"]
    assert "H out of range" in msgs["range"]
    assert "rank 1: device lost (planted)" in msgs["lost"]
    # the failed run appended only the sections before the failure and kept no checkpoint
    obs = pathlib.Path(lost) / "0.2500-obs.bin"
    assert obs.stat().st_size == NDIS * NREP * 11 * 4
    assert not (pathlib.Path(lost) / "0.2500-chkpt.bin").exists()


def test_cli_argument_errors(capsys):
    sys.path.insert(0, str(ROOT / "spin-glass_b200"))
    import csg_sharded
    assert csg_sharded.main([]) == 1 and "missing arguments" in capsys.readouterr().out
    assert csg_sharded.main(["a", "0", "x"]) == 1 and "extra arguments" in capsys.readouterr().out


@pytest.mark.gpu
def test_sharded_command_on_the_gpu_writes_the_single_gpu_commands_files(tmp_path):
    """Under torchrun (one rank, NCCL) the sharded command writes the same
    bytes as the single-GPU `csg` command for the same csg.conf."""
    import os
    import subprocess

    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    conf = dict(L=8, NDIS=64, NREP=8, SBSHFL=1, SBMEAS=64, SPFILE=128, seed=12345,
                beta_max=2.0, beta_min=0.5)
    a, b = pathlib.Path(_conf(tmp_path / "a", **conf)), pathlib.Path(_conf(tmp_path / "b", **conf))
    r = subprocess.run([str(ROOT / "spin-glass_b200" / "csg"), str(a), "0.25"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node=1", "--master-addr=127.0.0.1",
                        f"--master-port={_free_port()}",
                        str(ROOT / "spin-glass_b200" / "csg_sharded.py"), str(b), "0.25"],
                       cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for f in ("0.2500-obs.bin", "0.2500-chkpt.bin", "0.2500-chkpt.csg"):
        assert (a / f).read_bytes() == (b / f).read_bytes(), f
    assert not list(tmp_path.glob("*.log"))
