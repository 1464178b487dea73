"""csg_obs_records_noalloc: observable records for callers that cannot let a
library allocate device memory (their device memory all belongs to their own
pool or budget, where a library's cudaMalloc could fail and its cudaFree would
synchronise the device).  It must give the records of the allocating entry
point, csg_obs_records, call after call, with its fixed scratch array reused.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(csg):
    f = csg.lib().csg_obs_records_noalloc
    f.argtypes = [C.POINTER(csg.Config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                  C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("L,W,T,H", [
    (12, 2, 16, 0.0625),
    (24, 1, 8, 0.0),   # shared-memory and stride edge of the resident kernel sizes
    (32, 1, 4, 0.3),   # a streaming-engine lattice (L > 24)
])
def test_noalloc_records_match_allocating_entry_point(csg, L, W, T, H):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    betas = csg.geometric_betas(T, 0.5, 2.0)
    f = _entry(csg)
    with csg.Engine(L, W, 2, betas, H=H, seed=77, sweeps_per_swap=1) as e:
        e.init_lattice()
        for _call in range(2):  # two calls in a row: the scratch keeps the last contents
            e.run(6)
            want = e.obs_records()
            s, b, _ = e.get_state()
            ds = torch.from_numpy(s.view(np.int32)).cuda()
            db = torch.from_numpy(b.view(np.int32)).cuda()
            out = torch.full((32 * W, T, 11), float("nan"), dtype=torch.float32, device="cuda")
            rc = f(C.byref(e.cfg), ds.data_ptr(), db.data_ptr(), out.data_ptr(), out.numel(),
                   torch.cuda.current_stream().cuda_stream)
            assert rc == 0, csg.lib().csg_last_error().decode()
            torch.cuda.synchronize()
            # the same kernels and cos/sin table as csg_obs_records: equal bit for bit
            np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_noalloc_rejects_states_beyond_the_scratch(csg):
    f = _entry(csg)
    betas = csg.geometric_betas(64, 0.5, 2.0)
    cfg, _keep = csg.make_config(24, 64, 2, betas)
    n = 32 * 64 * 64 * 11
    rc = f(C.byref(cfg), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), n, None)
    assert rc == 3  # CSG_ERR_UNSUPPORTED, before any device access
    assert "16 MiB" in csg.lib().csg_last_error().decode()
