"""The C ABI boundary on CPU: the library loads and exports every symbol
include/dtwj.h declares, host-side argument checks, band rounding, error
strings and the CLI's argv behaviour.  No compute calls."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "dtwj.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(dtwj_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(dtwj):
    lib = dtwj.load()
    declared = _declared_symbols()
    assert set(declared) == set(dtwj.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_band_rounding(dtwj):
    assert dtwj.band(256, 0.01) == 3           # ceil(2.56)
    assert dtwj.band(1024, 0.05) == 52         # ceil(51.2)
    assert dtwj.band(1024, 0.05, "round") == 51
    assert dtwj.band(512, 0.2) == 103
    assert dtwj.band(512, 0.1) == 52
    assert dtwj.band(256, 0.05) == 13
    assert dtwj.band(32, 0.01, "round") == 1   # max(round(0.32), 1)
    assert dtwj.band(1000, 0.1) == 100         # exact products are not bumped


def test_error_strings(dtwj):
    for code in range(0, -11, -1):
        assert dtwj.strerror(code) not in ("", "unknown error")
    assert dtwj.strerror(-99) == "unknown error"


def test_argument_errors_are_reported_before_device_work(dtwj):
    x = np.zeros(100)
    for m, w in [(4, 1), (60, 3), (16, -1)]:
        with pytest.raises(dtwj.DtwjError) as e:
            dtwj.join(x, m, w)
        assert e.value.code == dtwj.ERR_ARG


def test_no_device_is_an_error_not_a_fallback(dtwj):
    if dtwj.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(dtwj.DtwjError) as e:
        dtwj.join(np.random.default_rng(0).standard_normal(500).cumsum(), 16, 2)
    assert e.value.code == dtwj.ERR_NODEVICE


def test_cli_unopenable_file_mirrors_reference(tmp_path):
    cli = os.path.join(PKG_DIR, "bin", "dtwj")
    r = subprocess.run([cli, str(tmp_path / "missing.txt"), str(tmp_path / "t.txt"), "64",
                        "0.05"], capture_output=True, text=True)
    # loadfile prints this and exits with status 0 (GPU_version1/src/loadfile.cu:17-21)
    assert r.returncode == 0
    assert "Error opening file" in r.stderr
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2
    # every documented option is accepted (parsed before the file is read);
    # an unknown one is refused
    for opt in ("--masked-cascade", "--petitjean", "--no-masked", "--no-seed", "--verbose",
                "--band-rounding=round", "--band=7", "--format=rows", "--json=" + str(tmp_path / "r.json")):
        r = subprocess.run([cli, str(tmp_path / "missing.txt"), str(tmp_path / "t.txt"), "64",
                            "0.05", opt], capture_output=True, text=True)
        assert r.returncode == 0 and "Error opening file" in r.stderr, opt
    r = subprocess.run([cli, str(tmp_path / "missing.txt"), str(tmp_path / "t.txt"), "64", "0.05",
                        "--no-such-option"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown option" in r.stderr


def test_lb_petitjean_argument_errors_before_device_work(dtwj):
    x = np.random.default_rng(1).standard_normal(3000).cumsum()
    s = 3000 - 64 + 1
    for m, w, a, b in [(64, 3, [0], [s]), (64, 3, [-1], [10]), (4, 3, [0], [10]),
                       (64, -1, [0], [100])]:
        with pytest.raises(dtwj.DtwjError) as e:
            dtwj.pair_lb_petitjean(x, m, w, a, b)
        assert e.value.code == dtwj.ERR_ARG, (m, w, a, b)
    # tables beyond the shared-memory limit: 2 (m + 2w) + 4m doubles > 200 KiB
    big = np.random.default_rng(2).standard_normal(40000).cumsum()
    with pytest.raises(dtwj.DtwjError) as e:
        dtwj.pair_lb_petitjean(big, 4200, 255, [0], [8400], own_env=True)
    assert e.value.code == dtwj.ERR_ARG


def test_synthetic_generators_are_deterministic(synth):
    a = synth.random_walk(1000, 3)
    b = synth.random_walk(1000, 3)
    assert a[0] == 0.0 and np.array_equal(a, b)
    e = synth.ecg_like(5000, 1)
    assert e.shape == (5000,) and np.isfinite(e).all()
    x = synth.random_walk(20000, 9)
    planted = synth.plant_motifs(x, 2, 256, 9)
    assert len(planted) == 2
    for a0, b0 in planted:
        assert abs(a0 - b0) >= 256
    assert synth.band(1024, 0.05) == 52
