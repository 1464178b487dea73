"""The result table on the GPU (csg_analyze_records) equals the host
restatement of analyze-all.py's estimators (spin-glass_b200/analysis.py) on
the same record file."""
import importlib

import numpy as np
import pytest


def _records(path, n_meas, ndis, nrep, seed):
    rng = np.random.default_rng(seed)
    an = importlib.import_module("spin_glass_b200.analysis")
    rec = np.zeros((n_meas, ndis, nrep), an.OBS_DT)
    rec["e"] = rng.uniform(-1.8, -0.2, (n_meas, ndis, nrep, 2))
    rec["m"] = rng.uniform(-0.2, 0.2, (n_meas, ndis, nrep, 2))
    # overlaps whose spread grows towards the cold end, as in a real run
    width = np.linspace(0.8, 0.05, nrep)
    rec["q_0"] = rng.normal(0, 1, (n_meas, ndis, nrep)) * width
    rec["q_1_r"] = rng.normal(0, 1, (n_meas, ndis, nrep, 3)) * width[:, None] * 0.3
    rec["q_1_i"] = rng.normal(0, 1, (n_meas, ndis, nrep, 3)) * width[:, None] * 0.3
    rec.tofile(path)


def test_analysis_entry_point_is_exported(csg):
    assert hasattr(csg.lib(), "csg_analyze_records")


@pytest.mark.gpu
@pytest.mark.parametrize("L,n_meas,ndis,nrep", [(16, 40, 64, 24), (8, 9, 300, 8)])
def test_gpu_table_equals_host_table(csg, tmp_path, L, n_meas, ndis, nrep):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    an = importlib.import_module("spin_glass_b200.analysis")
    path = str(tmp_path / "obs.bin")
    _records(path, n_meas, ndis, nrep, seed=L + ndis)
    host = an.analyze(path, L, ndis, nrep)
    gpu = an.analyze_gpu(path, L, ndis, nrep)
    assert gpu["n_meas"] == host["n_meas"] > 0
    for k in ("chi0", "chi0_err", "xi", "xi_err", "e", "e_err", "m", "m_err"):
        np.testing.assert_allclose(gpu[k], host[k], rtol=1e-11, atol=1e-15, err_msg=k)
