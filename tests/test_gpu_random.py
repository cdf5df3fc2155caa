"""Seeded random small relations (empty to dense; general, up-oriented and
symmetric; ids spread up to 2^24) through every device plan, compared with
the oracle exactly: the triangle, 4-clique, lollipop and barbell counts, both
selections for a few values, and the materialized triangle rows."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relation(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 160))
    m = int(rng.integers(0, 6 * n))
    kind = seed % 3
    u = rng.integers(0, n, m).astype(np.uint32)
    v = rng.integers(0, n, m).astype(np.uint32)
    if kind == 1:  # up-oriented without self-loops
        keep = u != v
        u, v = np.minimum(u, v)[keep], np.maximum(u, v)[keep]
    elif kind == 2:  # symmetric without self-loops
        keep = u != v
        u, v = u[keep], v[keep]
        u, v = np.concatenate([u, v]), np.concatenate([v, u])
    if seed % 5 == 0:  # spread ids (sparse sets, wide ranges)
        spread = np.sort(rng.choice(1 << 24, n, replace=False)).astype(np.uint32)
        u, v = spread[u], spread[v]
    return u, v, kind


@pytest.mark.parametrize("seed", range(60))
def test_random_relation_every_plan(eh, oracle, seed):
    u, v, kind = _relation(seed)
    ot = oracle.Trie(u, v)
    for policy, forced in ((0, 1), (2, 0), (2, 3)):
        t = eh.Trie(u, v, policy=policy, forced=forced, max_bitset_bytes=1 << 40)
        assert t.count("triangle") == ot.triangle(), (seed, policy, forced)
        assert t.count("lollipop") == ot.lollipop(), (seed, policy, forced)
        assert t.count("barbell") == ot.barbell(), (seed, policy, forced)
        assert t.count("clique4") == ot.clique4(), (seed, policy, forced)
        values = np.unique(np.concatenate([u, v]))
        for val in values[:: max(1, len(values) // 3)][:3]:
            assert t.count_select("barbell_sel", int(val)) == ot.barbell_sel(int(val)), (seed, val)
            assert t.count_select("clique4_sel", int(val)) == ot.clique4_sel(int(val)), (seed, val)
        rows = t.materialize()
        want = ot.triangle_tuples()
        if kind == 2:  # symmetric: the device writes each undirected triangle's 3! orderings; same set
            want = want[np.lexsort((want[:, 2], want[:, 1], want[:, 0]))]
        np.testing.assert_array_equal(rows, want)
        t.free()
