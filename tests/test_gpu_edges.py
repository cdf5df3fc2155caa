"""The device on the degenerate relations the oracle is pinned on against the
compiled reference engine (tests/test_oracle_edges.py): one row, a
self-loop, duplicates and both directions of a triangle, a 2-cycle, a
directed 3-cycle, complete graphs in one or both directions, a star, sparse
large ids.  Every COUNT plan, the 4-clique included on general relations
(self-loops, rows in both directions that are not symmetric), and both
selections at every value, under three layout policies; integer counts,
exact."""
import numpy as np
import pytest

from test_oracle_edges import CASES, PLANS

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CASES))
def test_degenerate_relations_on_the_device(eh, oracle, name):
    s, d = (np.array(x, np.uint32) for x in CASES[name])
    o = oracle.Trie(s, d)
    for policy, forced in ((0, 1), (2, 0), (2, 3)):
        t = eh.Trie(s, d, policy=policy, forced=forced, max_bitset_bytes=1 << 40)
        for mode in PLANS:
            assert t.count(mode) == getattr(o, mode)(), (name, mode, policy, forced)
        for v in np.unique(np.concatenate([s, d])).tolist():
            assert t.count_select("clique4_sel", v) == o.clique4_sel(v), (name, v)
            assert t.count_select("barbell_sel", v) == o.barbell_sel(v), (name, v)
        t.free()
