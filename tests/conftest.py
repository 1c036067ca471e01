"""Shared fixtures: the product (libdtwj.so through its Python binding), the
oracle (oracle/_build/liboracle.so, a C restatement of the reference) and the
reference itself (oracle/_ref/, built from the reference's own sources), plus
the golden fixtures under tests/golden/."""
from __future__ import annotations

import ctypes
import importlib.util
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "scaling-subsequence-similarity-join-based-on-dynamic-time-warping-cpu-gpu_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_join")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_package():
    if "dtwj" in sys.modules:
        return sys.modules["dtwj"]
    spec = importlib.util.spec_from_file_location(
        "dtwj", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dtwj"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_synth():
    spec = importlib.util.spec_from_file_location("dtwj_synth", os.path.join(PKG_DIR, "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class OrcResult(ctypes.Structure):
    _fields_ = [("i", ctypes.c_int64), ("j", ctypes.c_int64), ("dist", ctypes.c_double),
                ("seed_bsf", ctypes.c_double)] + [
        (k, ctypes.c_uint64) for k in ("pairs", "pruned_fast", "pruned_masked", "pruned_kim",
                                      "pruned_keogh", "dtw_calls", "dtw_abandoned")
    ] + [("seconds", ctypes.c_double), ("threads", ctypes.c_int)]


class Oracle:
    """ctypes view of oracle/dtwj_oracle.h (test infrastructure only)."""

    NO_DIAG, NO_MASKED, NO_SEED = 1, 2, 4

    def __init__(self, path=ORACLE_LIB):
        self.lib = ctypes.CDLL(path)
        P = ctypes.POINTER(ctypes.c_double)
        self.lib.orc_dtw2.restype = ctypes.c_double
        self.lib.orc_dtw2.argtypes = [P, P, ctypes.c_int, ctypes.c_int]
        self.lib.orc_pair_dist.restype = ctypes.c_double
        self.lib.orc_pair_dist.argtypes = [P, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int64, ctypes.c_int64]
        self.lib.orc_lb_keogh2.restype = ctypes.c_double

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def join(self, x, m, w, flags=0, threads=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        r = OrcResult()
        rc = self.lib.orc_join(self._p(x), ctypes.c_int64(x.size), m, w, flags, threads,
                               ctypes.byref(r))
        assert rc == 0, rc
        return r

    def dtw(self, q, t, w):
        q = np.ascontiguousarray(q, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        return float(np.sqrt(self.lib.orc_dtw2(self._p(q), self._p(t), q.size, w)))

    def pair_dist(self, x, m, w, i, j):
        x = np.ascontiguousarray(x, dtype=np.float64)
        return self.lib.orc_pair_dist(self._p(x), x.size, m, w, i, j)

    def stats(self, x, m):
        x = np.ascontiguousarray(x, dtype=np.float64)
        s = x.size - m + 1
        mu, sg = np.empty(s), np.empty(s)
        self.lib.orc_stats(self._p(x), ctypes.c_int64(x.size), m, self._p(mu), self._p(sg))
        return mu, sg

    def envelope(self, x, r):
        x = np.ascontiguousarray(x, dtype=np.float64)
        lo, up = np.empty(x.size), np.empty(x.size)
        self.lib.orc_envelope(self._p(x), ctypes.c_int64(x.size), r, self._p(lo), self._p(up))
        return lo, up

    def mp(self, x, m):
        x = np.ascontiguousarray(x, dtype=np.float64)
        s = x.size - m + 1
        mp, mpi = np.empty(s), np.empty(s, dtype=np.int64)
        self.lib.orc_mp(self._p(x), ctypes.c_int64(x.size), m, self._p(mp),
                        mpi.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        return mp, mpi

    def lb_petitjean(self, x, m, w, a, b, exact_env=True):
        """(keogh_full, keogh_mid, terms) of window a against window b."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        kf, km, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.lib.orc_lb_petitjean(self._p(x), ctypes.c_int64(x.size), m, w, ctypes.c_int64(a),
                                  ctypes.c_int64(b), int(bool(exact_env)), ctypes.byref(kf),
                                  ctypes.byref(km), ctypes.byref(t))
        return kf.value, km.value, t.value

    def kim2(self, q, t):
        q = np.ascontiguousarray(q, dtype=np.float64)
        t = np.ascontiguousarray(t, dtype=np.float64)
        left, right = ctypes.c_double(), ctypes.c_double()
        self.lib.orc_kim2(self._p(q), self._p(t), q.size, ctypes.byref(left), ctypes.byref(right))
        return left.value + right.value

    def mask(self, x, m, w):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.empty(x.size)
        lt = ctypes.c_int()
        rc = self.lib.orc_mask(self._p(x), ctypes.c_int64(x.size), m, w, self._p(out),
                               ctypes.byref(lt))
        assert rc == 0
        return out, lt.value


@pytest.fixture(scope="session")
def oracle():
    if not os.path.exists(ORACLE_LIB):
        pytest.skip("oracle not built (make -C oracle)")
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "joins.json")) as f:
        cases = json.load(f)
    for c in cases:
        c["series"] = np.fromfile(os.path.join(GOLDEN, "series_%s.f64" % c["name"]), dtype="<f8")
    return cases


@pytest.fixture(scope="session")
def kat():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def petitjean_kat():
    with open(os.path.join(GOLDEN, "petitjean.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def synth():
    return load_synth()


@pytest.fixture(scope="session")
def dtwj():
    return load_package()


@pytest.fixture(scope="session")
def gpu_dtwj(dtwj):
    if dtwj.device_count() < 1:
        pytest.fail("no CUDA device visible to libdtwj.so")
    return dtwj
