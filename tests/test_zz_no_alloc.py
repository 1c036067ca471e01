"""dtwj_pair_dtw_noalloc: the allocation-free pair DTW, for callers that must
not allocate device memory after start-up (a host framework that reserves the
device at initialisation, a latency-bound loop that cannot afford cudaMalloc's
implicit synchronisation).  It must give the same distances as the allocating
dtwj_pair_dtw, on two calls in a row (its fixed scratch is reused), allocate
nothing, write NaN for a pair whose index lies outside the series, accept the
largest series its scratch holds and refuse larger ones.  Collected last on
purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, xd, n, m, w, pid, pjd, count, precise, out):
    return lib.dtwj_pair_dtw_noalloc(ctypes.c_void_p(xd.data_ptr()), n, m, w,
                                     ctypes.c_void_p(pid.data_ptr()),
                                     ctypes.c_void_p(pjd.data_ptr()), count, precise,
                                     ctypes.c_void_p(out.data_ptr()), None)


def _pairs(n, m, count, seed):
    rng = np.random.default_rng(seed)
    pi = rng.integers(0, n - m + 1, count).astype(np.int64)
    pj = rng.integers(0, n - m + 1, count).astype(np.int64)
    return pi, pj


def test_no_alloc_pair_dtw_matches_allocating_entry_point(gpu_dtwj, synth):
    import torch

    lib = gpu_dtwj.load()
    x = synth.random_walk(30000, 123)
    n, m = x.size, 256
    count = 400
    pi, pj = _pairs(n, m, count, 9)
    xd = torch.from_numpy(x).cuda()
    pid = torch.from_numpy(pi).cuda()
    pjd = torch.from_numpy(pj).cuda()
    # same tolerances as the pair-DTW parity test: FP64 1e-10, FP32 2e-4;
    # w = 13 and w >= m (clamped to the full matrix on both entry points)
    for w in (13, 300):
        for precise, rtol in ((1, 1e-10), (0, 2e-4)):
            ref = gpu_dtwj.pair_dtw(x, m, w, pi, pj, precise=bool(precise))
            for _ in range(2):
                out = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda")
                rc = _call(lib, xd, n, m, w, pid, pjd, count, precise, out)
                torch.cuda.synchronize()
                assert rc == gpu_dtwj.OK, gpu_dtwj.strerror(rc)
                np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=rtol, atol=0)


def test_no_alloc_allocates_nothing(gpu_dtwj, synth):
    import torch

    lib = gpu_dtwj.load()
    x = synth.random_walk(20000, 5)
    n, m, w = x.size, 128, 7
    pi, pj = _pairs(n, m, 256, 3)
    xd = torch.from_numpy(x).cuda()
    pid = torch.from_numpy(pi).cuda()
    pjd = torch.from_numpy(pj).cuda()
    out = torch.empty(256, dtype=torch.float64, device="cuda")
    assert _call(lib, xd, n, m, w, pid, pjd, 256, 0, out) == gpu_dtwj.OK  # warm
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for precise in (0, 1, 0):
        assert _call(lib, xd, n, m, w, pid, pjd, 256, precise, out) == gpu_dtwj.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_no_alloc_out_of_range_index_gives_nan(gpu_dtwj, synth):
    import torch

    lib = gpu_dtwj.load()
    x = synth.random_walk(8000, 11)
    n, m, w = x.size, 100, 6
    s = n - m + 1
    pi, pj = _pairs(n, m, 64, 4)
    ref = gpu_dtwj.pair_dtw(x, m, w, pi, pj, precise=True)
    bad = pi.copy()
    bad[5] = s          # one past the last window
    bad[17] = -1
    xd = torch.from_numpy(x).cuda()
    out = torch.zeros(64, dtype=torch.float64, device="cuda")
    rc = _call(lib, xd, n, m, w, torch.from_numpy(bad).cuda(), torch.from_numpy(pj).cuda(), 64,
               1, out)
    torch.cuda.synchronize()
    assert rc == gpu_dtwj.OK
    got = out.cpu().numpy()
    assert np.isnan(got[5]) and np.isnan(got[17])
    keep = np.ones(64, dtype=bool)
    keep[[5, 17]] = False
    np.testing.assert_allclose(got[keep], ref[keep], rtol=1e-10, atol=0)


def test_no_alloc_size_limits(gpu_dtwj, synth):
    import torch

    lib = gpu_dtwj.load()
    m = 64
    n = gpu_dtwj.NOALLOC_MAX_WINDOWS + m - 1  # exactly the windows the scratch holds
    x = synth.random_walk(n, 13)
    xd = torch.from_numpy(x).cuda()
    pi = np.array([0, n - m, 1000], dtype=np.int64)
    pj = np.array([n - m, 5000, 200000], dtype=np.int64)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _call(lib, xd, n, m, 3, torch.from_numpy(pi).cuda(), torch.from_numpy(pj).cuda(), 3, 1,
               out)
    torch.cuda.synchronize()
    assert rc == gpu_dtwj.OK, gpu_dtwj.strerror(rc)
    np.testing.assert_allclose(out.cpu().numpy(), gpu_dtwj.pair_dtw(x, m, 3, pi, pj, precise=True),
                               rtol=1e-10, atol=0)
    # one window too many: refused before any launch
    big = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    idx = torch.zeros(1, dtype=torch.int64, device="cuda")
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _call(lib, big, n + 1, m, 3, idx, idx, 1, 1, one)
    assert rc == gpu_dtwj.ERR_SCRATCH
    assert "scratch" in gpu_dtwj.strerror(rc)
    # m beyond the library's limit: an argument error, as for dtwj_pair_dtw
    rc = _call(lib, big, n + 1, 70000, 3, idx, idx, 1, 1, one)
    assert rc == gpu_dtwj.ERR_ARG
