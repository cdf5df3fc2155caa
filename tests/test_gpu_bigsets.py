"""Sets larger than one warp's share of the layout build (the head set of a
large relation, hubs of a symmetric one) are built grid-wide: their
reference-format bytes and the counts over them must not change.
Integer work: exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BITSET, UINT, BLOCK = 0, 1, 3


def norm_bitset(raw):
    raw = np.array(raw, np.uint8)
    w = (len(raw) - 8) // 12
    words = raw[8: 8 + 8 * w].view(np.uint64)
    rank = raw[8 + 8 * w: 8 + 12 * w].view(np.uint32).copy()
    rank[words == 0] = 0
    return np.concatenate([raw[: 8 + 8 * w], rank.view(np.uint8)])


def _relation(seed=11):
    """Three hub rows with 10,000-45,000 children over a dense range (bitset
    by the density rule), many small rows, and a head set of ~70,000."""
    rng = np.random.default_rng(seed)
    src, dst = [], []
    for hub, n, span in ((5, 60000, 100000), (70001, 12000, 30000), (123456, 30000, 3_000_000)):
        d = np.unique(rng.integers(0, span, n)).astype(np.uint32)
        src.append(np.full(len(d), hub, np.uint32))
        dst.append(d)
    a = rng.integers(0, 140000, 400000).astype(np.uint32)
    b = rng.integers(0, 140000, 400000).astype(np.uint32)
    src.append(a)
    dst.append(b)
    s = np.concatenate(src)
    d = np.concatenate(dst)
    keep = s != d
    return s[keep], d[keep]


@pytest.mark.parametrize("policy,forced", [(0, UINT), (2, BITSET), (2, BLOCK)], ids=["heuristic", "bitset", "block"])
def test_big_set_bytes_and_counts(eh, oracle, policy, forced):
    s, d = _relation()
    ot = oracle.Trie(s, d)
    t = eh.Trie(s, d, policy=policy, forced=forced, max_bitset_bytes=1 << 50)
    lens = np.diff(ot.off)
    big = [int(i) for i in np.nonzero(lens > 8192)[0]]
    assert len(big) == 3
    for i in big + [None]:
        raw, lay = t.set_bytes(i)
        elems = ot.head if i is None else ot.child(i)
        if lay == BITSET:
            np.testing.assert_array_equal(norm_bitset(raw), norm_bitset(oracle.range_bitset(elems)))
        elif lay == BLOCK:
            np.testing.assert_array_equal(raw, oracle.block_bitset(elems))
        else:
            np.testing.assert_array_equal(raw.view(np.uint32), elems)
    assert t.count("triangle") == ot.triangle()
