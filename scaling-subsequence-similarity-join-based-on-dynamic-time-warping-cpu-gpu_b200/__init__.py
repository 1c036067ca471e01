"""dtwj: B200-native top-1 z-normalised DTW subsequence self-join.

Python binding over the C ABI of lib/libdtwj.so (include/dtwj.h).  The
library is the product; this module only marshals arrays.  Loading fails
loudly when the shared library is missing: there is no CPU fallback.

Reference seam mirrored here: ``DTWMotifDiscoveryGUI(TS, subseqlen, maxwarp,
output_time_file_path)`` (CPU_version1/DTWMotifDiscoveryGUI.cpp:12) runs the
ED matrix profile and the join, prints the result and appends the join time
to the file; :func:`dtw_motif_discovery` does the same and also returns the
result.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdtwj.so")
CLI_PATH = os.path.join(_HERE, "bin", "dtwj")

OK = 0
ERR_ARG = -1
ERR_NAN = -2
ERR_CUDA = -3
ERR_OOM = -4
ERR_BAND = -5
ERR_OVERFLOW = -6
ERR_TIMEOUT = -7
ERR_NODEVICE = -8
ERR_IO = -9
ERR_NOMODEL = -10
ERR_SCRATCH = -11
NOALLOC_MAX_WINDOWS = 262144

F_NO_MASKED = 0x1
F_NO_SEED = 0x2
F_NO_DIAG = 0x4
F_LEARNED = 0x8
F_VERBOSE = 0x10
F_PROFILE = 0x20
F_NO_GRAPH = 0x40
F_MASKED_CASCADE = 0x80
F_PETITJEAN = 0x100

PHASES = ("prep", "profile", "seeds", "diag", "pairs", "verify", "runs", "keogh")

# Every symbol include/dtwj.h declares.
EXPORTS = (
    "dtwj_join",
    "dtwj_join_batch",
    "dtwj_ctx_create",
    "dtwj_ctx_destroy",
    "dtwj_ctx_join",
    "dtwj_ctx_join_device",
    "dtwj_matrix_profile",
    "dtwj_global_mask",
    "dtwj_pair_dtw",
    "dtwj_pair_lb_petitjean",
    "dtwj_pair_dtw_noalloc",
    "dtwj_band",
    "dtwj_strerror",
    "dtwj_device_count",
    "dtwj_mlp_create",
    "dtwj_mlp_destroy",
    "dtwj_mlp_get",
    "dtwj_mlp_set",
    "dtwj_mlp_train",
    "dtwj_mlp_predict",
    "dtwj_mlp_grad",
    "dtwj_mlp_save",
    "dtwj_mlp_load",
    "dtwj_ctx_set_model",
    "dtwj_ctx_tiles",
    "dtwj_band_shapes",
    "dtwj_time_band",
    "dtwj_ctx_set_band",
    "dtwj_ctx_set_tuning",
    "dtwj_ctx_set_shard",
    "dtwj_ctx_set_exchange",
    "dtwj_load",
)

LOAD_FORMATS = {"values": 0, "every": 1, "first-column": 2, "rows": 3, "binary": 4}

MLP_IN = 64
MLP_HIDDEN = 128
MLP_PARAMS = 24961


class DtwjError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__("%s%s (code %d)" % (what + ": " if what else "", strerror(code), code))


class _Result(ctypes.Structure):
    _fields_ = [
        ("i", ctypes.c_int64),
        ("j", ctypes.c_int64),
        ("dist", ctypes.c_double),
        ("dist_fp32", ctypes.c_double),
        ("seed_bsf", ctypes.c_double),
        ("pairs", ctypes.c_uint64),
        ("pruned_fast", ctypes.c_uint64),
        ("pruned_kim", ctypes.c_uint64),
        ("pruned_masked", ctypes.c_uint64),
        ("pruned_keogh", ctypes.c_uint64),
        ("dtw_calls", ctypes.c_uint64),
        ("dtw_abandoned", ctypes.c_uint64),
        ("dtw_cells", ctypes.c_uint64),
        ("candidates", ctypes.c_uint64),
        ("seconds_join", ctypes.c_double),
        ("seconds_total", ctypes.c_double),
        ("n", ctypes.c_int64),
        ("m", ctypes.c_int32),
        ("w", ctypes.c_int32),
        ("phase_seconds", ctypes.c_double * 8),
        ("phase_launches", ctypes.c_uint64 * 8),
        ("pruned_paa", ctypes.c_uint64),
        ("pruned_petitjean", ctypes.c_uint64),
    ]


@dataclass
class JoinResult:
    i: int
    j: int
    dist: float
    dist_fp32: float
    seed_bsf: float
    pairs: int
    pruned_fast: int
    pruned_kim: int
    pruned_masked: int
    pruned_keogh: int
    dtw_calls: int
    dtw_abandoned: int
    dtw_cells: int
    candidates: int
    seconds_join: float
    seconds_total: float
    n: int
    m: int
    w: int
    phase_seconds: list
    phase_launches: list
    pruned_paa: int
    pruned_petitjean: int = 0

    @staticmethod
    def _from(r: _Result) -> "JoinResult":
        d = {}
        for name, _ in _Result._fields_:
            v = getattr(r, name)
            d[name] = list(v) if name.startswith("phase_") else v
        return JoinResult(**d)


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libdtwj.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libdtwj.so not built at %s (run build.py)" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    d = ctypes.c_double
    i32, i64, u32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
    lib.dtwj_join.argtypes = [P(d), i64, i32, i32, u32, P(_Result)]
    lib.dtwj_join_batch.argtypes = [P(P(d)), P(i64), P(i32), P(i32), i32, u32, P(_Result)]
    lib.dtwj_ctx_create.argtypes = [ctypes.c_int, P(ctypes.c_void_p)]
    lib.dtwj_ctx_destroy.argtypes = [ctypes.c_void_p]
    lib.dtwj_ctx_destroy.restype = None
    lib.dtwj_ctx_join.argtypes = [ctypes.c_void_p, P(d), i64, i32, i32, u32, P(_Result)]
    lib.dtwj_ctx_join_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, i64, i32, i32, u32,
                                         P(_Result)]
    lib.dtwj_matrix_profile.argtypes = [P(d), i64, i32, P(d), P(i64)]
    lib.dtwj_global_mask.argtypes = [P(d), i64, i32, i32, P(ctypes.c_float), P(i32)]
    lib.dtwj_pair_dtw.argtypes = [P(d), i64, i32, i32, P(i64), P(i64), i64, i32, P(d)]
    lib.dtwj_pair_lb_petitjean.argtypes = [P(d), i64, i32, i32, P(i64), P(i64), i64, i32, P(d),
                                           P(d)]
    vp = ctypes.c_void_p
    lib.dtwj_pair_dtw_noalloc.argtypes = [vp, i64, i32, i32, vp, vp, i64, i32, vp, vp]
    lib.dtwj_band.argtypes = [i32, d, i32]
    lib.dtwj_band.restype = i32
    lib.dtwj_strerror.argtypes = [ctypes.c_int]
    lib.dtwj_strerror.restype = ctypes.c_char_p
    lib.dtwj_device_count.argtypes = []
    f32p = P(ctypes.c_float)
    lib.dtwj_mlp_create.argtypes = [ctypes.c_int, ctypes.c_uint64, P(vp)]
    lib.dtwj_mlp_destroy.argtypes = [vp]
    lib.dtwj_mlp_destroy.restype = None
    lib.dtwj_mlp_get.argtypes = [vp, f32p]
    lib.dtwj_mlp_set.argtypes = [vp, f32p]
    lib.dtwj_mlp_train.argtypes = [vp, f32p, f32p, i64, i32, i32, ctypes.c_float,
                                   ctypes.c_uint64, f32p]
    lib.dtwj_mlp_predict.argtypes = [vp, f32p, i64, f32p]
    lib.dtwj_mlp_grad.argtypes = [vp, f32p, f32p, i64, i32, f32p, f32p]
    lib.dtwj_mlp_save.argtypes = [vp, ctypes.c_char_p]
    lib.dtwj_mlp_load.argtypes = [ctypes.c_int, ctypes.c_char_p, P(vp)]
    lib.dtwj_ctx_set_model.argtypes = [vp, vp]
    lib.dtwj_band_shapes.argtypes = [i32, P(i32), P(i32), i32]
    lib.dtwj_time_band.argtypes = [ctypes.c_int, i32, i32, i32, i32, i32, P(d)]
    lib.dtwj_ctx_set_band.argtypes = [vp, i32, i32, i32]
    lib.dtwj_ctx_set_tuning.argtypes = [vp, i32, i32]
    lib.dtwj_ctx_set_shard.argtypes = [vp, i32, i32]
    lib.dtwj_ctx_set_exchange.argtypes = [vp, EXCHANGE_FN, vp, i32]
    lib.dtwj_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i32, i32, P(d), i64, P(i64)]
    lib.dtwj_ctx_tiles.argtypes = [vp, P(d), i64, i32, i32, P(i64), P(i32), f32p, P(d)]
    _lib = lib
    return lib


def _f64(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def strerror(code: int) -> str:
    return load().dtwj_strerror(code).decode()


def device_count() -> int:
    return int(load().dtwj_device_count())


def band(m: int, ratio: float, rounding: str = "ceil") -> int:
    return int(load().dtwj_band(m, ratio, 1 if rounding == "round" else 0))


def join(x, m: int, w: int, flags: int = 0) -> JoinResult:
    """Top-1 z-normalised DTW pair of x (j - i >= m, band w)."""
    a = _f64(x)
    r = _Result()
    rc = load().dtwj_join(_dptr(a), a.size, m, w, flags, ctypes.byref(r))
    if rc != OK:
        raise DtwjError(rc, "dtwj_join")
    return JoinResult._from(r)


def join_batch(series, ms, ws, flags: int = 0) -> list[JoinResult]:
    """Top-1 pair of each series (dtwj_join_batch): the series of one (m, w)
    are joined together in one pass, up to four such groups at the same time
    on device 0; each result equals join(series[k], ms[k], ws[k], flags)."""
    arrs = [_f64(x) for x in series]
    k = len(arrs)
    ptrs = (ctypes.POINTER(ctypes.c_double) * k)(*[_dptr(a) for a in arrs])
    ns = (ctypes.c_int64 * k)(*[a.size for a in arrs])
    mm = (ctypes.c_int32 * k)(*ms)
    ww = (ctypes.c_int32 * k)(*ws)
    outs = (_Result * k)()
    rc = load().dtwj_join_batch(ptrs, ns, mm, ww, k, flags, outs)
    if rc != OK:
        raise DtwjError(rc, "dtwj_join_batch")
    return [JoinResult._from(outs[q]) for q in range(k)]


# void fn(void* user, uint32_t* bsf2_dev, int32_t count, void* stream)
EXCHANGE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                               ctypes.c_void_p)


class _DeviceWords:
    """__cuda_array_interface__ view of count int32 words at a device address
    (the context's best-so-far: float bits of non-negative squared distances,
    which order like the floats and stay below 2^31)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4",
                                         "data": (ptr, False), "version": 3}


def bsf_allreduce(words, group=None):
    """Lowers every shard's best-so-far words (an int32 tensor of float bits)
    to their minimum over the process group, in place."""
    import torch.distributed as dist
    dist.all_reduce(words, op=dist.ReduceOp.MIN, group=group)


def make_exchange(group=None, device: int | None = None):
    """Exchange callback for Context.set_exchange: an all-reduce(min) of the
    best-so-far words over the group (NCCL), enqueued on the join's stream."""
    import torch

    def exchange(user, ptr, count, stream):
        words = torch.as_tensor(_DeviceWords(ptr, count),
                                device="cuda" if device is None else "cuda:%d" % device)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            bsf_allreduce(words, group)
    return exchange


class Context:
    """Reusable device context (keeps device buffers between joins).

    tune_cache: a JSON file written by autotune.tune_join (default: the
    DTWJ_TUNE_CACHE environment variable, if set).  Before the first join of
    an (m, w) the context applies that file's entry for it, if there is one;
    it never tunes by itself."""

    def __init__(self, device: int = 0, tune_cache: str | None = None):
        lib = load()
        h = ctypes.c_void_p()
        rc = lib.dtwj_ctx_create(device, ctypes.byref(h))
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_create")
        self._h = h
        self._tune_cache = tune_cache if tune_cache is not None else os.environ.get("DTWJ_TUNE_CACHE")
        self._tuned = set()

    def _apply_tuning(self, m: int, w: int):
        if not self._tune_cache or (m, w) in self._tuned:
            return
        self._tuned.add((m, w))
        from . import autotune
        e = autotune.load_cache(self._tune_cache).get(autotune.join_key(m, w))
        if e:
            autotune.apply_entry(self, m, w, e)

    def close(self):
        if self._h:
            load().dtwj_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def join(self, x, m: int, w: int, flags: int = 0) -> JoinResult:
        self._apply_tuning(m, w)
        a = _f64(x)
        r = _Result()
        rc = load().dtwj_ctx_join(self._h, _dptr(a), a.size, m, w, flags, ctypes.byref(r))
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_join")
        return JoinResult._from(r)

    def set_shard(self, rank: int, world: int):
        """Join only the tiles t with t % world == rank (dtwj_ctx_set_shard)."""
        rc = load().dtwj_ctx_set_shard(self._h, rank, world)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_set_shard")

    def set_exchange(self, fn, phases: int = 8):
        """Sharded joins sweep in `phases` groups and call fn(user, bsf2_ptr,
        count, stream_ptr) after each (dtwj_ctx_set_exchange); None removes it."""
        cb = EXCHANGE_FN(fn) if fn is not None else EXCHANGE_FN()
        rc = load().dtwj_ctx_set_exchange(self._h, cb, None, phases if fn is not None else 0)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_set_exchange")
        self._exchange = cb  # the library holds the pointer: keep the thunk alive

    def set_band(self, w: int, C: int = 0, G: int = 0):
        """Joins with band w use the DTW layout (C cells per lane, G lanes per
        pair); (0, 0) restores the default choice."""
        rc = load().dtwj_ctx_set_band(self._h, w, C, G)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_set_band")

    def set_tuning(self, dtw_warps: int = 0, chunk_tiles: int = 0):
        """CTA size of the DTW kernel in warps (1, 2, 4, 8) and tiles per chunk
        of the diagonal sweep (16..4096); 0 restores a default."""
        rc = load().dtwj_ctx_set_tuning(self._h, dtw_warps, chunk_tiles)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_set_tuning")

    def set_model(self, net):
        """Network used by joins with F_LEARNED on this context (None clears)."""
        rc = load().dtwj_ctx_set_model(self._h, net._h if net is not None else None)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_set_model")
        self._model = net  # keep it alive while the context may use it

    def tiles(self, x, m: int, w: int, features: bool = True, min_dist: bool = False):
        """(desc [T][4] = (first lag, first row, rows, lags), features [T][64] or
        None, min_dist [T] or None) for the diagonal-sweep tiles of x."""
        a = _f64(x)
        cnt = ctypes.c_int64()
        lib = load()
        rc = lib.dtwj_ctx_tiles(self._h, _dptr(a), a.size, m, w, ctypes.byref(cnt), None, None,
                                None)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_tiles")
        t = cnt.value
        desc = np.empty((t, 4), dtype=np.int32)
        feat = np.empty((t, MLP_IN), dtype=np.float32) if features else None
        md = np.empty(t, dtype=np.float64) if min_dist else None
        rc = lib.dtwj_ctx_tiles(self._h, _dptr(a), a.size, m, w, ctypes.byref(cnt),
                                desc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                _fptr(feat) if feat is not None else None,
                                _dptr(md) if md is not None else None)
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_tiles")
        return desc, feat, md

    def join_device(self, dev_ptr: int, n: int, m: int, w: int, flags: int = 0) -> JoinResult:
        """Join a series already in device memory (dev_ptr: n float64)."""
        self._apply_tuning(m, w)
        r = _Result()
        rc = load().dtwj_ctx_join_device(self._h, ctypes.c_void_p(dev_ptr), n, m, w, flags,
                                         ctypes.byref(r))
        if rc != OK:
            raise DtwjError(rc, "dtwj_ctx_join_device")
        return JoinResult._from(r)


def matrix_profile(x, m: int):
    """(mp, mpi): z-normalised ED matrix profile, exclusion zone m."""
    a = _f64(x)
    s = a.size - m + 1
    mp = np.empty(max(s, 0), dtype=np.float64)
    mpi = np.empty(max(s, 0), dtype=np.int64)
    rc = load().dtwj_matrix_profile(_dptr(a), a.size, m, _dptr(mp),
                                    mpi.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if rc != OK:
        raise DtwjError(rc, "dtwj_matrix_profile")
    return mp, mpi


def global_mask(x, m: int, w: int):
    """(mask, table_len): the masked diagonal bound's global CDF mask (0/1 per
    sample) and its CDF table length, computed on the device."""
    a = _f64(x)
    out = np.empty(a.size, dtype=np.float32)
    lt = ctypes.c_int32()
    rc = load().dtwj_global_mask(_dptr(a), a.size, m, w,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                 ctypes.byref(lt))
    if rc != OK:
        raise DtwjError(rc, "dtwj_global_mask")
    return out, lt.value


def pair_dtw(x, m: int, w: int, pi, pj, precise: bool = True) -> np.ndarray:
    """Banded DTW distances of the z-normalised subsequence pairs (pi[k], pj[k])."""
    a = _f64(x)
    pi = np.ascontiguousarray(pi, dtype=np.int64)
    pj = np.ascontiguousarray(pj, dtype=np.int64)
    out = np.empty(pi.size, dtype=np.float64)
    P64 = ctypes.POINTER(ctypes.c_int64)
    rc = load().dtwj_pair_dtw(_dptr(a), a.size, m, w, pi.ctypes.data_as(P64),
                              pj.ctypes.data_as(P64), pi.size, 1 if precise else 0, _dptr(out))
    if rc != OK:
        raise DtwjError(rc, "dtwj_pair_dtw")
    return out


def pair_lb_petitjean(x, m: int, w: int, pa, pb, own_env: bool = False):
    """The two sums LB_Petitjean adds to the endpoint bound for windows
    pa[k] (A) against pb[k] (B): (keogh_mid, terms), FP64 on the device.
    own_env: each window's own clipped envelope (the reference's); else the
    raw series' envelope normalised per window (what DTWJ_F_PETITJEAN joins
    read)."""
    a = _f64(x)
    pa = np.ascontiguousarray(pa, dtype=np.int64)
    pb = np.ascontiguousarray(pb, dtype=np.int64)
    km = np.empty(pa.size, dtype=np.float64)
    tt = np.empty(pa.size, dtype=np.float64)
    P64 = ctypes.POINTER(ctypes.c_int64)
    rc = load().dtwj_pair_lb_petitjean(_dptr(a), a.size, m, w, pa.ctypes.data_as(P64),
                                       pb.ctypes.data_as(P64), pa.size, 1 if own_env else 0,
                                       _dptr(km), _dptr(tt))
    if rc != OK:
        raise DtwjError(rc, "dtwj_pair_lb_petitjean")
    return km, tt


def dtw_motif_discovery(ts, subseqlen: int, maxwarp: int, output_time_file_path: str,
                        flags: int = 0, quiet: bool = False) -> JoinResult:
    """Mirror of DTWMotifDiscoveryGUI (CPU_version1/DTWMotifDiscoveryGUI.cpp:12):
    join, print the reference's result lines (1-based indices), append the
    join time as "%lf\\n" to output_time_file_path."""
    r = join(ts, subseqlen, maxwarp, flags)
    if not quiet:
        print("first min is %d sec min is %d" % (r.i + 1, r.j + 1))
        print("total time is %fs   input of bsf:%5.3f  ,final distance :%f  "
              % (r.seconds_join, r.seed_bsf, r.dist))
    with open(output_time_file_path, "a") as f:
        f.write("%f\n" % r.seconds_join)
    return r


def _f32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class MLP:
    """Tile-scoring network of the learned ordering (dtwj_mlp_*): 64 -> 128 ->
    128 -> 1, BF16 tensor-core GEMMs with FP32 accumulation, Adam."""

    def __init__(self, device: int = 0, seed: int = 0, _handle=None):
        if _handle is None:
            h = ctypes.c_void_p()
            rc = load().dtwj_mlp_create(device, seed, ctypes.byref(h))
            if rc != OK:
                raise DtwjError(rc, "dtwj_mlp_create")
            _handle = h
        self._h = _handle

    @classmethod
    def load_file(cls, path: str, device: int = 0) -> "MLP":
        h = ctypes.c_void_p()
        rc = load().dtwj_mlp_load(device, path.encode(), ctypes.byref(h))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_load")
        return cls(_handle=h)

    def close(self):
        if self._h:
            load().dtwj_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.empty(MLP_PARAMS, dtype=np.float32)
        rc = load().dtwj_mlp_get(self._h, _fptr(p))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_get")
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        assert p.size == MLP_PARAMS
        rc = load().dtwj_mlp_set(self._h, _fptr(p))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_set")

    def train(self, x, y, epochs: int = 1, batch: int = 4096, lr: float = 1e-3,
              seed: int = 0) -> float:
        x = _f32(x).reshape(-1, MLP_IN)
        y = _f32(y).reshape(-1)
        loss = ctypes.c_float()
        rc = load().dtwj_mlp_train(self._h, _fptr(x), _fptr(y), x.shape[0], epochs, batch, lr,
                                   seed, ctypes.byref(loss))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_train")
        return loss.value

    def predict(self, x) -> np.ndarray:
        x = _f32(x).reshape(-1, MLP_IN)
        out = np.empty(x.shape[0], dtype=np.float32)
        rc = load().dtwj_mlp_predict(self._h, _fptr(x), x.shape[0], _fptr(out))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_predict")
        return out

    def grad(self, x, y, precise: bool = False):
        """(gradient in the parameter layout, loss) of the mean squared error."""
        x = _f32(x).reshape(-1, MLP_IN)
        y = _f32(y).reshape(-1)
        g = np.empty(MLP_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        rc = load().dtwj_mlp_grad(self._h, _fptr(x), _fptr(y), x.shape[0], 1 if precise else 0,
                                  _fptr(g), ctypes.byref(loss))
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_grad")
        return g, loss.value

    def save(self, path: str):
        rc = load().dtwj_mlp_save(self._h, path.encode())
        if rc != OK:
            raise DtwjError(rc, "dtwj_mlp_save")


def band_shapes(w: int) -> list:
    """[(C, G), ...]: the DTW layouts the autotuner tries for band w."""
    C = (ctypes.c_int32 * 16)()
    G = (ctypes.c_int32 * 16)()
    k = load().dtwj_band_shapes(w, C, G, 16)
    if k < 0:
        raise DtwjError(k, "dtwj_band_shapes")
    return [(C[q], G[q]) for q in range(min(k, 16))]


def time_band(m: int, w: int, C: int, G: int, pairs: int = 2048, device: int = 0) -> float:
    """Band cells per second of exact FP32 DTW with layout (C, G)."""
    v = ctypes.c_double()
    rc = load().dtwj_time_band(device, m, w, C, G, pairs, ctypes.byref(v))
    if rc != OK:
        raise DtwjError(rc, "dtwj_time_band")
    return v.value


_COUNTERS = ("pairs", "pruned_fast", "pruned_kim", "pruned_masked", "pruned_paa", "pruned_keogh",
             "pruned_petitjean", "dtw_calls",
             "dtw_abandoned", "dtw_cells", "candidates")


def merge_results(results) -> JoinResult:
    """One join's result from its shards' results: the lexicographic minimum
    of (dist, i, j) (a shard without a pair, i = -1, never wins), counters
    summed, times the maximum, seed_bsf the minimum."""
    rs = list(results)
    have = [r for r in rs if r.i >= 0]
    best = min(have, key=lambda r: (r.dist, r.i, r.j)) if have else rs[0]
    d = dict(best.__dict__)
    for k in _COUNTERS:
        d[k] = sum(getattr(r, k) for r in rs)
    d["seconds_join"] = max(r.seconds_join for r in rs)
    d["seconds_total"] = max(r.seconds_total for r in rs)
    d["seed_bsf"] = min(r.seed_bsf for r in rs)
    d["phase_seconds"] = [max(v) for v in zip(*(r.phase_seconds for r in rs))]
    d["phase_launches"] = [sum(v) for v in zip(*(r.phase_launches for r in rs))]
    return JoinResult(**d)


def join_sharded(x, m: int, w: int, flags: int = 0, device: int | None = None, group=None,
                 result_fn=None, exchange_phases: int = 8) -> JoinResult:
    """One join spread over the ranks of a torch.distributed process group:
    rank r sweeps the tiles t with t % world == r on its device (default: the
    current CUDA device).  With exchange_phases > 0 the ranks lower each
    other's best-so-far after each of that many sweep phases (an all-reduce
    of one word, make_exchange); at the end they exchange their results (one
    all_gather of a few numbers).  result_fn(rank, world) replaces the device
    join (tests of the exchange without a GPU)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if result_fn is not None:
        mine = result_fn(rank, world)
    else:
        if device is None:
            import torch
            device = torch.cuda.current_device()
        with Context(device) as ctx:
            ctx.set_shard(rank, world)
            if exchange_phases > 0 and world > 1:
                ctx.set_exchange(make_exchange(group, device), exchange_phases)
            mine = ctx.join(x, m, w, flags)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine.__dict__, group=group)
    return merge_results(JoinResult(**g) for g in gathered)


def load_series(path: str, fmt: str = "values", every: int = 1, path2: str | None = None):
    """A series file in one of the reference's formats (dtwj_load): "values"
    (loadfile), "every" (loadfile_apart, every `every`-th value), "first-column"
    (loadfile_2: first number of each line of path, then path2), "rows"
    (loadfile_: lines flattened row by row) or "binary" (raw float64)."""
    lib = load()
    n = ctypes.c_int64()
    p1, p2 = path.encode(), (path2.encode() if path2 else None)
    f = LOAD_FORMATS[fmt]
    rc = lib.dtwj_load(p1, p2, f, every, None, 0, ctypes.byref(n))
    if rc != OK:
        raise DtwjError(rc, "dtwj_load")
    out = np.empty(n.value, dtype=np.float64)
    rc = lib.dtwj_load(p1, p2, f, every, _dptr(out), out.size, ctypes.byref(n))
    if rc != OK:
        raise DtwjError(rc, "dtwj_load")
    return out
