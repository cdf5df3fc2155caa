"""Rule descriptors (eh_rule_match, host only): the reference's COUNT rules
(test/graph/travis.py) map to the device plans up to renaming and reordering
of their atoms; other bodies are refused."""
import itertools

import pytest

RULES = {
    "TriangleAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),z:long<-[COUNT(*)].": "triangle",
    "FliqueAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,d),Edge(b,d),Edge(c,d),z:long<-[COUNT(*)].": "clique4",
    "LollipopAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,x),z:long<-[COUNT(*)].": "lollipop",
    "BarbellAgg(;w) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,x),Edge(x,y),Edge(y,z),Edge(x,z),"
    "w:long<-[COUNT(*)].": "barbell",
    "FliqueSelAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,d),Edge(b,d),Edge(c,d),Edge(a,x),x=0,"
    "z:long<-[COUNT(*)].": "clique4_sel",
    "BarbellSelAgg(;w) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,p),Edge(p,x),Edge(x,y),Edge(y,z),Edge(x,z),p=6,"
    "w:long<-[COUNT(*)].": "barbell_sel",
}


@pytest.mark.parametrize("rule", list(RULES), ids=list(RULES.values()))
def test_reference_rules_match_their_plans(rule):
    from emptyheaded_b200 import datalog
    assert datalog.plan(rule) == RULES[rule]


def test_renamed_and_reordered_bodies():
    from emptyheaded_b200 import datalog
    for perm in itertools.permutations(["Edge(u,v)", "Edge(v,w)", "Edge(u,w)"]):
        assert datalog.plan("T(;n) :- %s,n:long<-[COUNT(*)]." % ",".join(perm)) == "triangle"
    body = "Edge(q,r),Edge(r,s),Edge(q,s),Edge(q,t),Edge(r,t),Edge(s,t),Edge(q,k),k=5"
    assert datalog.plan("F(;n) :- %s,n:long<-[COUNT(*)]." % body) == "clique4_sel"
    # a repeated atom is the same constraint
    assert datalog.plan("T(;n) :- Edge(a,b),Edge(b,c),Edge(a,c),Edge(a,b),n:long<-[COUNT(*)].") == "triangle"


@pytest.mark.parametrize("rule", [
    "C(;n) :- Edge(a,b),Edge(b,c),Edge(c,a),n:long<-[COUNT(*)].",          # directed 3-cycle
    "P(;n) :- Edge(a,b),Edge(b,c),n:long<-[COUNT(*)].",                     # 2-path
    "T(;n) :- Edge(a,b),Other(b,c),Edge(a,c),n:long<-[COUNT(*)].",          # two relations
    "S(;n) :- Edge(a,b),Edge(b,c),Edge(a,c),b=3,n:long<-[COUNT(*)].",       # selection on a triangle
])
def test_other_bodies_are_refused(rule):
    import emptyheaded_b200 as E
    from emptyheaded_b200 import datalog
    with pytest.raises(E.EHError):
        datalog.plan(rule, relation_names=("Edge", "Other"))


def test_parser_refuses_what_it_cannot_count():
    from emptyheaded_b200 import datalog
    for bad in ["Triangle(a,b,c) :- Edge(a,b),Edge(b,c),Edge(a,c).",     # materialized head
                "T(;z) :- Edge(a,b),Edge(b,c),Edge(a,c).",                # no aggregate
                "T(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),z:long<-[SUM(a;1)]."]:
        with pytest.raises(ValueError):
            datalog.parse(bad)
