"""Golden outputs of the reference's own series loaders (CPU_version1/loadfile.cpp:
loadfile, loadfile_apart, loadfile_2, loadfile_) on the sample files in
tests/golden/loaders/, through the oracle shim (oracle/_ref/libref.so, built by
oracle/build_ref.sh from the reference tree).  Writes tests/golden/loaders.json.

    python tests/golden/make_loader_golden.py
"""
import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")

# (name, format, param, file, file2): format 0 loadfile, 1 loadfile_apart,
# 2 loadfile_2, 3 loadfile_
CASES = [
    ("values", 0, 0, "values.txt", None),
    ("every_1", 1, 1, "values.txt", None),
    ("every_3", 1, 3, "values.txt", None),
    ("first_column_2", 2, 0, "col_a.txt", "col_b.txt"),
    ("rows", 3, 0, "matrix.txt", None),
]


def main():
    lib = ctypes.CDLL(LIB)
    lib.ref_load.restype = ctypes.c_long
    lib.ref_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_double), ctypes.c_long]
    out = []
    for name, fmt, param, f1, f2 in CASES:
        p1 = os.path.join(HERE, "loaders", f1).encode()
        p2 = os.path.join(HERE, "loaders", f2).encode() if f2 else None
        buf = (ctypes.c_double * 256)()
        k = lib.ref_load(p1, p2, fmt, param, buf, 256)
        out.append(dict(name=name, format=fmt, param=param, file=f1, file2=f2,
                        values=[buf[q] for q in range(min(k, 256))]))
    with open(os.path.join(HERE, "loaders.json"), "w") as f:
        json.dump(out, f, indent=1)
    for c in out:
        print(c["name"], c["values"])


if __name__ == "__main__":
    main()
