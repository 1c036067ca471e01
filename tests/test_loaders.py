"""Series loaders (dtwj_load, CPU): every format against the reference's own
loaders' outputs on the sample files (tests/golden/loaders.json, made by
tests/golden/make_loader_golden.py), plus the cases the reference does not
handle (unreadable file, ragged matrix, binary)."""
import json
import os

import numpy as np
import pytest

from conftest import load_package

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FORMATS = {0: "values", 1: "every", 2: "first-column", 3: "rows"}


def test_loaders_match_the_reference():
    dtwj = load_package()
    cases = json.load(open(os.path.join(HERE, "loaders.json")))
    assert len(cases) == 5
    for c in cases:
        p1 = os.path.join(HERE, "loaders", c["file"])
        p2 = os.path.join(HERE, "loaders", c["file2"]) if c["file2"] else None
        x = dtwj.load_series(p1, FORMATS[c["format"]], every=max(c["param"], 1), path2=p2)
        np.testing.assert_array_equal(x, np.array(c["values"]), err_msg=c["name"])


def test_loader_errors_and_binary(tmp_path):
    dtwj = load_package()
    with pytest.raises(dtwj.DtwjError) as e:
        dtwj.load_series(str(tmp_path / "missing.txt"))
    assert e.value.code == dtwj.ERR_IO
    rag = tmp_path / "ragged.txt"
    rag.write_text("1 2 3\n4 5\n")
    with pytest.raises(dtwj.DtwjError) as e:
        dtwj.load_series(str(rag), "rows")
    assert e.value.code == dtwj.ERR_IO
    with pytest.raises(dtwj.DtwjError) as e:
        dtwj.load_series(str(rag), "every", every=0)
    assert e.value.code == dtwj.ERR_ARG
    x = np.random.default_rng(3).normal(size=1001)
    b = tmp_path / "x.f64"
    x.astype("<f8").tofile(b)
    np.testing.assert_array_equal(dtwj.load_series(str(b), "binary"), x)
    # one file for the first-column format
    assert list(dtwj.load_series(os.path.join(HERE, "loaders", "col_b.txt"), "first-column")) == [9.0, 11.25, 12.0]
