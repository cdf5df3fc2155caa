"""Materialized triangle output on the device against the reference's
goldens (test/graph/travis.py:282-318) and the oracle's listing (exact
tuples, exact order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_triangle_rows_facebook(eh, oracle, facebook):
    p = facebook["pruned"]
    t = eh.Trie(p[:, 0], p[:, 1])
    rows = t.materialize()
    assert rows.shape == (1612010, 3) and tuple(rows[0]) == (6, 5, 2)
    np.testing.assert_array_equal(rows, oracle.Trie(p[:, 0], p[:, 1]).triangle_tuples())
    proj = t.materialize(project=True)
    assert proj.shape == (85658, 2) and tuple(proj[0]) == (6, 5)
    np.testing.assert_array_equal(proj, oracle.Trie(p[:, 0], p[:, 1]).triangle_projection())
    t.free()


@pytest.mark.parametrize("kind", ["duplicated", "simple", "general", "up"])
def test_triangle_rows_match_oracle(eh, oracle, facebook, kind):
    if kind in ("duplicated", "simple"):
        a = facebook[kind]
        s, d = a[:, 0], a[:, 1]
    elif kind == "general":
        rng = np.random.default_rng(5)
        s = rng.integers(0, 200, 4000).astype(np.uint32)
        d = rng.integers(0, 200, 4000).astype(np.uint32)
    else:
        u, v = oracle.gen_rmat(3, 12, 16 << 12)
        s, d, _ = oracle.preprocess(u, v)
    for policy, forced in ((0, 1), (2, 0), (2, 3)):
        t = eh.Trie(s, d, policy=policy, forced=forced)
        np.testing.assert_array_equal(t.materialize(), oracle.Trie(s, d).triangle_tuples())
        t.free()
