"""eh_query_weighted_root: the lollipop / barbell root bags over an arbitrary
annotated unary relation z (by value), against a numpy restatement of the
root bags (sum_a z(a)|N(a)| and sum over rows (a,x) of z(a)z(x), modulo
2^64), on an up-oriented, a symmetric and a general relation; z covers
values outside the head, values beyond the array, and large values that wrap."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _want(s, d, z, query):
    zv = lambda v: np.where(v < len(z), z[np.minimum(v, len(z) - 1)], 0).astype(np.uint64)
    rows = np.unique(np.stack([s, d], 1), axis=0)
    a, x = rows[:, 0].astype(np.int64), rows[:, 1].astype(np.int64)
    with np.errstate(over="ignore"):
        if query == "lollipop":
            return int((zv(a) * np.uint64(1)).sum(dtype=np.uint64))
        return int((zv(a) * zv(x)).sum(dtype=np.uint64))


@pytest.mark.parametrize("kind", ["up", "symmetric", "general"])
def test_weighted_root_matches_restatement(eh, oracle, kind):
    rng = np.random.default_rng(17)
    if kind == "up":
        u, v = oracle.gen_rmat(3, 12, 16 << 12)
        s, d, _ = oracle.preprocess(u, v)
    elif kind == "symmetric":
        u, v = oracle.gen_rmat(5, 11, 16 << 11)
        s, d, _ = oracle.preprocess(u, v, symmetric=True)
    else:
        s = rng.integers(0, 500, 6000).astype(np.uint32)
        d = rng.integers(0, 500, 6000).astype(np.uint32)
    n = int(max(s.max(), d.max())) + 1
    t = eh.Trie(s, d)
    for size in (n, n // 2, n + 10):
        z = rng.integers(0, 1 << 62, size, dtype=np.uint64)  # products wrap modulo 2^64
        for q in ("lollipop", "barbell"):
            assert t.weighted_root(q, z) == _want(s, d, z, q), (kind, size, q)
    t.free()
