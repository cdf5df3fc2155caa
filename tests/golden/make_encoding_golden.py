"""Writes encoding.npz: the reference's own Encoding<T> (Encoding.cpp:21-48,
run through oracle/_ref/eh_ref encode) on seeded columns of each numeric
value type it instantiates (uint32_t, int, long, float).

    python tests/golden/make_encoding_golden.py   (needs the reference checkout, $EH_REFERENCE or ../reference, and
                                                   oracle/_ref/eh_ref)

Per type: three columns sharing one encoding (the loader encodes every
column of an attribute type together, createDB.scala:242-270), with
duplicates, the type's extremes and, for float, negative values, +-inf and
-0.0 beside +0.0."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def columns(value_type, seed):
    rng = np.random.default_rng(seed)
    dt = O.VALUE_TYPES[value_type][1]
    if value_type == "uint32":
        a = rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(dt)
        b = rng.integers(0, 5000, 8000).astype(dt)            # dense, repeated
        c = np.array([0, 0xFFFFFFFF, 7, 7, 5000], dt)
    elif value_type == "int32":
        a = rng.integers(-(1 << 31), 1 << 31, 5000, dtype=np.int64).astype(dt)
        b = rng.integers(-3000, 3000, 8000).astype(dt)
        c = np.array([-(1 << 31), (1 << 31) - 1, 0, -1, 1], dt)
    elif value_type == "int64":
        a = rng.integers(-(1 << 62), 1 << 62, 5000, dtype=np.int64).astype(dt)
        b = rng.integers(-3000, 3000, 8000).astype(dt)
        c = np.array([np.iinfo(np.int64).min, np.iinfo(np.int64).max, 0, -1, 1], dt)
    else:
        a = (rng.standard_normal(5000) * 1e6).astype(dt)
        b = rng.integers(-50, 50, 8000).astype(dt) / np.float32(4)
        c = np.array([np.inf, -np.inf, 0.0, -0.0, 1.5, -1.5, np.finfo(np.float32).tiny], dt)
    return [a, b, c]


def main():
    out = {}
    for i, vt in enumerate(O.VALUE_TYPES):
        cols = columns(vt, 100 + i)
        values, keys = O.ref_encoding(cols, vt)
        out[vt + "_values"] = values
        for j, (c, k) in enumerate(zip(cols, keys)):
            out["%s_col%d" % (vt, j)] = c
            out["%s_keys%d" % (vt, j)] = k
        print(vt, "distinct", len(values))
    np.savez_compressed(os.path.join(HERE, "encoding.npz"), **out)


if __name__ == "__main__":
    main()
