"""dtwj_pair_dtw_noalloc: the allocation-free pair DTW, for callers that must
not allocate device memory after start-up (a host framework that reserves the
device at initialisation, a latency-bound loop that cannot afford cudaMalloc's
implicit synchronisation).  It must give the same distances as the allocating
dtwj_pair_dtw, on two calls in a row (its fixed scratch is reused), and must
refuse series larger than that scratch.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, xd, n, m, w, pid, pjd, count, precise, out):
    return lib.dtwj_pair_dtw_noalloc(ctypes.c_void_p(xd.data_ptr()), n, m, w,
                                     ctypes.c_void_p(pid.data_ptr()),
                                     ctypes.c_void_p(pjd.data_ptr()), count, precise,
                                     ctypes.c_void_p(out.data_ptr()), None)


def test_no_alloc_pair_dtw_matches_allocating_entry_point(gpu_dtwj, synth):
    import torch

    lib = gpu_dtwj.load()
    x = synth.random_walk(30000, 123)
    n, m, w = x.size, 256, 13
    rng = np.random.default_rng(9)
    count = 400
    pi = rng.integers(0, n - m + 1, count).astype(np.int64)
    pj = rng.integers(0, n - m + 1, count).astype(np.int64)
    xd = torch.from_numpy(x).cuda()
    pid = torch.from_numpy(pi).cuda()
    pjd = torch.from_numpy(pj).cuda()
    # same tolerances as the pair-DTW parity test: FP64 1e-10, FP32 2e-4
    for precise, rtol in ((1, 1e-10), (0, 2e-4)):
        ref = gpu_dtwj.pair_dtw(x, m, w, pi, pj, precise=bool(precise))
        for _ in range(2):
            out = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda")
            rc = _call(lib, xd, n, m, w, pid, pjd, count, precise, out)
            torch.cuda.synchronize()
            assert rc == gpu_dtwj.OK, gpu_dtwj.strerror(rc)
            np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=rtol, atol=0)


def test_no_alloc_rejects_series_beyond_its_scratch(gpu_dtwj):
    import torch

    lib = gpu_dtwj.load()
    m = 64
    n = gpu_dtwj.NOALLOC_MAX_WINDOWS + m  # one window too many
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    idx = torch.zeros(1, dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _call(lib, xd, n, m, 3, idx, idx, 1, 1, out)
    assert rc == gpu_dtwj.ERR_SCRATCH
    assert "scratch" in gpu_dtwj.strerror(rc)
