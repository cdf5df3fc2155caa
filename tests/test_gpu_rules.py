"""eh_rule_count through the reference's own COUNT rules (test/graph/travis.py)
on its graphs: the counts its tests assert."""
import pytest

pytestmark = pytest.mark.gpu

PRUNED = {
    "TriangleAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),z:long<-[COUNT(*)].": ("triangle", 1612010),
    "FliqueAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,d),Edge(b,d),Edge(c,d),z:long<-[COUNT(*)].":
        ("clique4", 30004668),
}
DUPLICATED = {
    "LollipopAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,x),z:long<-[COUNT(*)].": ("lollipop", 1426911480),
    "BarbellAgg(;w) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,x),Edge(x,y),Edge(y,z),Edge(x,z),w:long<-[COUNT(*)].":
        ("barbell", 20371831447136),
    "FliqueSelAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,d),Edge(b,d),Edge(c,d),Edge(a,x),x=0,"
    "z:long<-[COUNT(*)].": ("clique4_sel", 3759972),
    "BarbellSelAgg(;w) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,p),Edge(p,x),Edge(x,y),Edge(y,z),Edge(x,z),p=6,"
    "w:long<-[COUNT(*)].": ("barbell_sel", 26936100),
}


@pytest.mark.parametrize("graph,rules", [("pruned", PRUNED), ("duplicated", DUPLICATED)])
def test_travis_rules(eh, facebook, graph, rules):
    from emptyheaded_b200 import datalog
    a = facebook[graph]
    t = eh.Trie(a[:, 0], a[:, 1])
    for rule, (plan, want) in rules.items():
        c, st = datalog.count(rule, {"Edge": t}, stats=True)
        assert (st["plan"], c) == (plan, want), rule
    t.free()


def test_rule_over_a_second_relation(eh, facebook):
    """Atoms name the relation they read: the triangle over Other is counted
    on the trie given as Other."""
    from emptyheaded_b200 import datalog
    p = facebook["pruned"]
    d = facebook["duplicated"]
    t1, t2 = eh.Trie(d[:, 0], d[:, 1]), eh.Trie(p[:, 0], p[:, 1])
    assert datalog.count("T(;n) :- Other(a,b),Other(b,c),Other(a,c),n:long<-[COUNT(*)].",
                         {"Edge": t1, "Other": t2}) == 1612010
