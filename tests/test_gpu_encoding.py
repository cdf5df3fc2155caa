"""Device dictionary encoding (eh_encoding_*) against the reference's own
Encoding<T> (Encoding.cpp:21-48; fixture tests/golden/encoding.npz) and the
oracle.  Integer keys and bit patterns of values: exact."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("vt", ["uint32", "int32", "int64", "float32"])
def test_encoding_matches_reference(eh, vt):
    z = np.load(os.path.join(GOLDEN, "encoding.npz"))
    cols = [z["%s_col%d" % (vt, j)] for j in range(3)]
    enc = eh.Encoding(cols, vt)
    want = z[vt + "_values"]
    assert len(enc) == len(want)
    assert enc.values().tobytes() == want.tobytes()
    for j, c in enumerate(cols):
        keys = enc.encode(c)
        np.testing.assert_array_equal(keys, z["%s_keys%d" % (vt, j)])
        dec = enc.decode(keys)
        # decode(encode(x)) == x, with -0.0 read back as the encoding's zero
        np.testing.assert_array_equal(dec, c)
    enc.free()


def test_encoding_large_dense_and_sparse(eh, oracle):
    """A dense id domain (dense map) and a sparse one (binary search) at a
    few million values: keys equal the oracle's."""
    rng = np.random.default_rng(7)
    dense = [rng.integers(0, 1 << 21, 3_000_000).astype(np.uint32), np.arange(1 << 20, dtype=np.uint32)]
    sparse = [rng.integers(0, 1 << 32, 3_000_000, dtype=np.uint64).astype(np.uint32)]
    for cols in (dense, sparse):
        enc = eh.Encoding(cols, "uint32")
        values, keys = oracle.encoding(cols, "uint32")
        np.testing.assert_array_equal(enc.values(), values)
        for c, k in zip(cols, keys):
            np.testing.assert_array_equal(enc.encode(c), k)
        enc.free()


def test_encoding_errors(eh):
    enc = eh.Encoding([np.array([3, 1, 2], np.uint32)], "uint32")
    with pytest.raises(eh.EHError):
        enc.encode(np.array([4], np.uint32))      # value_to_key.at throws
    with pytest.raises(eh.EHError):
        enc.decode(np.array([3], np.uint32))      # key out of range
    with pytest.raises(eh.EHError):
        eh.Encoding([np.array([1.0, np.nan], np.float32)], "float32")
    np.testing.assert_array_equal(enc.encode(np.array([1, 2, 3], np.uint32)), [0, 1, 2])


def test_encoded_relation_counts(eh, facebook, golden):
    """Encode facebook_pruned with a gap-spread id space (values * 1000 + 17),
    build the trie from the keys: the triangle count is the reference's."""
    p = facebook["pruned"].astype(np.uint64) * 1000 + 17
    enc = eh.Encoding([p[:, 0], p[:, 1]], "int64")
    s, d = enc.encode(p[:, 0].astype(np.int64)), enc.encode(p[:, 1].astype(np.int64))
    t = eh.Trie(s, d)
    assert t.count("triangle") == golden["travis"]["facebook_pruned"]["triangle"]
