"""The `csg <sim_dir> <H>` command: the reference program's interface
(Program/src/main.cu:8-84), its files, and a bit-exact resume."""
import os
import pathlib
import shutil
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
CLI = ROOT / "spin-glass_b200" / "csg"
# The reference checkout: $CSG_REFERENCE_ROOT, else a directory "reference"
# beside this repository (tests that need it skip when it is absent).
REFERENCE = pathlib.Path(os.environ.get("CSG_REFERENCE_ROOT", str(ROOT.parent / "reference")))


def run_cli(args, cwd):
    return subprocess.run([str(CLI), *args], cwd=cwd, capture_output=True, text=True, timeout=600)


def write_conf(d: pathlib.Path, **kv):
    d.mkdir(parents=True, exist_ok=True)
    (d / "csg.conf").write_text("".join(f"{k} = {v}\n" for k, v in kv.items()))


def test_argument_errors(tmp_path):
    assert CLI.exists()
    r = run_cli([], tmp_path)
    assert r.returncode == 1 and "missing arguments" in r.stdout
    r = run_cli(["a", "0", "x"], tmp_path)
    assert r.returncode == 1 and "extra arguments" in r.stdout


def test_field_out_of_range_fails_and_keeps_log(tmp_path):
    r = run_cli([str(tmp_path), "4.5"], tmp_path)
    assert r.returncode == 1 and "H out of range" in r.stdout
    assert list(tmp_path.glob("*.log")), "the log is kept on failure (main.cu:70-75)"


OBS_DT = np.dtype([("e", "f4", (2,)), ("m", "f4", (2,)), ("q_0", "f4"), ("q_1_r", "f4", (3,)),
                   ("q_1_i", "f4", (3,))])


@pytest.mark.skipif(not (REFERENCE / "analyze-all.py").exists(),
                    reason="the reference's analyze-all.py is not on this machine")
def test_reference_analysis_reads_our_records_unchanged(orc, tmp_path):
    """Records laid out exactly as the engine writes them (oracle-made here)
    go through the reference's own analyze-all.py, unmodified."""
    sim = tmp_path / "Simulations"
    for L, H in [(12, 0.0), (14, 0.0), (16, 0.0), (16, 0.0625), (16, 0.125), (16, 0.1875)]:
        d = sim / f"{L:02d}"
        d.mkdir(parents=True, exist_ok=True)
        recs = []
        for section in range(2):
            spins, bonds = orc.init(L, 64, 2, 24, 100 * L + section)
            recs.append(orc.obs_records(spins, bonds, L, H))
        data = np.concatenate(recs).astype(np.float32)
        assert data.shape == (2 * 2048, 24, 11)
        data.tofile(d / f"{H:06.4f}-obs.bin")
        assert np.fromfile(d / f"{H:06.4f}-obs.bin", dtype=OBS_DT).shape == (2 * 2048 * 24,)
    r = subprocess.run([sys.executable, str(REFERENCE / "analyze-all.py")], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = (sim / "16" / "0.0000-res.dat").read_text().splitlines()
    assert res[0].startswith("# tot_MC_steps : 2,048")
    rows = np.array([[float(v) for v in ln.split()] for ln in res[1:]])
    assert rows.shape == (24, 9)
    np.testing.assert_allclose(rows[:, 0], np.logspace(1, -3, 24, base=2.0))
    # the chunked restatement (spin-glass_b200/analysis.py) gives the same tables
    # (it accumulates in float64 where analyze-all.py averages float32 arrays)
    sys.path.insert(0, str(ROOT / "spin-glass_b200"))
    import analysis
    for L, H in [(12, 0.0), (16, 0.1875)]:
        mine = tmp_path / f"mine-{L}-{H}.dat"
        analysis.write_table(analysis.analyze(str(sim / f"{L:02d}" / f"{H:06.4f}-obs.bin"), L,
                                              2048, 24, chunk=1), str(mine))
        want = (sim / f"{L:02d}" / f"{H:06.4f}-res.dat").read_text().splitlines()
        got = mine.read_text().splitlines()
        assert got[0] == want[0]
        np.testing.assert_allclose(np.array([[float(v) for v in ln.split()] for ln in got[1:]]),
                                   np.array([[float(v) for v in ln.split()] for ln in want[1:]]),
                                   rtol=1e-3, atol=1e-9)


# ---------------------------------------------------------------- on the GPU
small = dict(L=8, NDIS=64, NREP=8, SBSHFL=1, SBMEAS=64, seed=12345, beta_max=2.0, beta_min=0.5)


@pytest.mark.gpu
def test_run_writes_reference_files_and_matches_oracle(orc, tmp_path):
    d = tmp_path / "sim"
    write_conf(d, SPFILE=256, **small)
    r = run_cli([str(d), "0.25"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert not list(tmp_path.glob("*.log")), "the log is removed on success (main.cu:77-80)"
    obs = np.fromfile(d / "0.2500-obs.bin", dtype=np.float32).reshape(4, 64, 8, 11)
    chk = np.fromfile(d / "0.2500-chkpt.bin", dtype=np.uint32).reshape(128, 512)
    assert (d / "0.2500-chkpt.csg").read_text().split() == ["csg-resume-v1", "256", "12345"]
    # the same chain on the oracle
    L, T = 8, 8
    ratio = (0.5 / 2.0) ** (1.0 / (T - 1))
    betas = np.array([np.float32(ratio ** r * 2.0) for r in range(T)], np.float64)
    spins, bonds = orc.init(L, 2, 2, T, 12345)
    for sec in range(4):
        orc.run(spins, bonds, L=L, betas=betas, H=0.25, seed=12345, sweep0=64 * sec, n_sweeps=64,
                sweeps_per_swap=1)
        np.testing.assert_array_equal(obs[sec], orc.obs_records(spins, bonds, L, 0.25))
    np.testing.assert_array_equal(chk, orc.to_ref_lattice(spins, bonds, L))


@pytest.mark.gpu
def test_resume_is_bit_exact(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    write_conf(a, SPFILE=128, **small)
    write_conf(b, SPFILE=256, **small)
    for _ in range(2):
        assert run_cli([str(a), "0"], tmp_path).returncode == 0
    assert run_cli([str(b), "0"], tmp_path).returncode == 0
    assert (a / "0.0000-obs.bin").read_bytes() == (b / "0.0000-obs.bin").read_bytes()
    assert (a / "0.0000-chkpt.bin").read_bytes() == (b / "0.0000-chkpt.bin").read_bytes()
    assert (a / "0.0000-chkpt.csg").read_text() == (b / "0.0000-chkpt.csg").read_text()


@pytest.mark.gpu
def test_reference_checkpoint_without_sidecar_starts_a_new_chain(tmp_path):
    d = tmp_path / "sim"
    write_conf(d, SPFILE=64, **small)
    assert run_cli([str(d), "0"], tmp_path).returncode == 0
    (d / "0.0000-chkpt.csg").unlink()
    r = run_cli([str(d), "0"], tmp_path)
    assert r.returncode == 0 and "checkpoint loaded" in r.stdout
    assert (d / "0.0000-obs.bin").stat().st_size == 2 * 64 * 8 * 44


@pytest.mark.gpu
def test_truncated_checkpoint_fails(tmp_path):
    d = tmp_path / "sim"
    write_conf(d, SPFILE=64, **small)
    assert run_cli([str(d), "0"], tmp_path).returncode == 0
    data = (d / "0.0000-chkpt.bin").read_bytes()
    (d / "0.0000-chkpt.bin").write_bytes(data[:-4])
    r = run_cli([str(d), "0"], tmp_path)
    assert r.returncode == 1 and "truncated" in r.stdout
