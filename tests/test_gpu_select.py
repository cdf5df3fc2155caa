"""Equality-selection COUNT plans on the device (eh_query_count_select)
against the reference's asserted counts (test/graph/travis.py:385-401,
472-487) and the compiled reference engine's selection bags.  Integer
work: every comparison is exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UINT, BITSET, BLOCK = 1, 0, 3
POLICIES = [("heuristic", 0, 1), ("uint", 2, UINT), ("bitset", 2, BITSET), ("block", 2, BLOCK)]


def _trie(eh, s, d, policy, forced):
    return eh.Trie(np.ascontiguousarray(s, np.uint32), np.ascontiguousarray(d, np.uint32), policy=policy,
                   forced=forced, max_bitset_bytes=1 << 50)


@pytest.mark.parametrize("pol", POLICIES, ids=[p[0] for p in POLICIES])
def test_travis_selection_goldens(eh, facebook, golden, pol):
    """FliqueSelAgg x=0 -> 3759972, BarbellSelAgg p=6 -> 26936100 on
    facebook_duplicated, under every layout policy."""
    d = facebook["duplicated"]
    t = _trie(eh, d[:, 0], d[:, 1], pol[1], pol[2])
    tr = golden["travis"]["facebook_duplicated"]
    assert t.count_select("clique4_sel", 0) == tr["clique4_sel_x0"] == 3759972
    assert t.count_select("barbell_sel", 6) == tr["barbell_sel_p6"] == 26936100


@pytest.mark.parametrize("name", ["facebook_duplicated", "facebook_pruned", "rmat_s12_ef16_s3",
                                  "rmat_s14_ef16_s5_sym", "er_16384_131072_s1"])
def test_selection_vs_reference_engine(eh, oracle, facebook, golden, name):
    """Every selected value the reference engine was run with (low, middle
    and highest-degree nodes), on oriented and symmetric relations."""
    if name.startswith("facebook"):
        a = facebook[name.split("_")[1]]
        s, d = a[:, 0], a[:, 1]
    else:
        from test_oracle import _gen
        (u, v), sym = _gen(oracle, name)
        s, d, _ = oracle.preprocess(u, v, symmetric=sym)
    for pol in (POLICIES[0], POLICIES[2]):
        t = _trie(eh, s, d, pol[1], pol[2])
        for key, want in golden["select"][name].items():
            mode, val = key.rsplit("_", 1)
            assert t.count_select(mode, int(val)) == want, (pol[0], key)


def test_selection_matches_oracle_at_scale(eh, oracle):
    """R-MAT scale 16 (oriented) and scale 14 symmetric: device selection
    counts equal the oracle's for a spread of selected values."""
    for scale, seed, sym in ((16, 42, False), (14, 5, True)):
        u, v = oracle.gen_rmat(seed, scale, 16 << scale)
        s, d, nn = oracle.preprocess(u, v, symmetric=sym)
        ot = oracle.Trie(s, d)
        t = _trie(eh, s, d, 0, 1)
        for val in (0, nn // 7, nn // 3, nn - 2, nn - 1):
            assert t.count_select("clique4_sel", val) == ot.clique4_sel(val), (scale, val)
            assert t.count_select("barbell_sel", val) == ot.barbell_sel(val), (scale, val)


def test_selection_value_not_in_relation(eh):
    """A value in neither column fails like the reference's
    Encoding::value_to_key.at; a value only in the second column has no
    child set and counts 0 for the barbell (N(v) empty)."""
    s = np.array([0, 0, 1, 1, 2], np.uint32)
    d = np.array([1, 2, 2, 3, 3], np.uint32)
    t = eh.Trie(s, d)
    with pytest.raises(eh.EHError):
        t.count_select("clique4_sel", 9)
    with pytest.raises(eh.EHError):
        t.count_select("barbell_sel", 1 << 30)
    assert t.count_select("barbell_sel", 3) == 0
    # 4-cliques rooted at partners of 3 ({1, 2}): none in this relation
    assert t.count_select("clique4_sel", 3) == 0
