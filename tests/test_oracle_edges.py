"""The oracle against the compiled reference engine on degenerate relations:
one row, a self-loop, duplicates and both directions of a triangle, a
2-cycle, a directed 3-cycle, complete graphs stored in one or both
directions, a star, and sparse large ids; all four COUNT plans and both
selection plans at every value of the relation.  Integer counts: exact.  The
empty relation and a selected value absent from the relation are checked
against the oracle alone (0): the reference driver refuses an edge file with
no rows and a value its dictionary has no key for."""
import numpy as np
import pytest


def _complete(n, both):
    s, d = [], []
    for i in range(n):
        for j in range(n):
            if i != j and (both or i < j):
                s.append(i)
                d.append(j)
    return s, d


CASES = {
    "one_row": ([3], [7]),
    "self_loop": ([5], [5]),
    "triangle_mixed": ([0, 0, 1, 1, 1, 2, 0], [1, 2, 2, 2, 1, 0, 1]),
    "two_cycle": ([0, 1], [1, 0]),
    "directed_cycle": ([0, 1, 2], [1, 2, 0]),
    "k4_both_directions": _complete(4, True),
    "k5_upward": _complete(5, False),
    "star": ([0] * 50 + list(range(1, 51)), list(range(1, 51)) + [0] * 50),
    "far_ids": ([1000000, 1000000, 2000000], [2000000, 3000000, 3000000]),
}
PLANS = ("triangle", "clique4", "lollipop", "barbell")


@pytest.mark.parametrize("name", sorted(CASES))
def test_degenerate_relations_vs_reference_engine(oracle, name):
    if not oracle.ref_available():
        pytest.skip("reference engine not built")
    s, d = (np.array(x, np.uint32) for x in CASES[name])
    t = oracle.Trie(s, d)
    for mode in PLANS:
        want = oracle.ref_query_edges(mode, s, d, timeout=120)["count_u64"]
        assert getattr(t, mode)() == want, mode
    for v in np.unique(np.concatenate([s, d])).tolist():
        assert t.clique4_sel(v) == oracle.ref_query_edges("clique4_sel", s, d, timeout=120, value=v)["count_u64"], v
        assert t.barbell_sel(v) == oracle.ref_query_edges("barbell_sel", s, d, timeout=120, value=v)["count_u64"], v
    # a value absent from the relation selects nothing (the reference driver
    # refuses it: the dictionary has no key for it)
    absent = int(max(s.max(), d.max())) + 1
    assert t.clique4_sel(absent) == 0 and t.barbell_sel(absent) == 0


def test_empty_relation(oracle):
    t = oracle.Trie(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    for mode in PLANS:
        assert getattr(t, mode)() == 0, mode
