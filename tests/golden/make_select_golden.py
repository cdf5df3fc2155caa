"""Adds the equality-selection queries to golden.json.

    python tests/golden/make_select_golden.py   (needs the reference checkout, $EH_REFERENCE or ../reference, and
                                                 oracle/_ref/eh_ref; run
                                                 after make_golden.py)

travis.select: the counts the reference's tests assert for
FliqueSelAgg (x=0) and BarbellSelAgg (p=6) on facebook_duplicated
(test/graph/travis.py:385-401, 472-487).
select: counts of the compiled reference engine (selection bags in
oracle/ref_driver.cpp) on the in-repo graphs and on seeded synthetic
graphs, for a few selection values each: a low-degree node, a middle node
and the highest-degree node (node ids are degree-ordered after
preprocessing)."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle import oracle as O  # noqa: E402
from test_oracle import _gen  # noqa: E402

GRAPHS = ["rmat_s12_ef16_s3", "rmat_s14_ef16_s5_sym", "er_16384_131072_s1"]


def values_for(nodes):
    return sorted({1, nodes // 2, nodes - 1})


def main():
    path = os.path.join(HERE, "golden.json")
    with open(path) as f:
        golden = json.load(f)
    golden["travis"]["facebook_duplicated"]["clique4_sel_x0"] = 3759972
    golden["travis"]["facebook_duplicated"]["barbell_sel_p6"] = 26936100
    fb = np.load(os.path.join(HERE, "facebook.npz"))
    out = {}
    for key in ("duplicated", "pruned"):
        a = fb[key]
        ent = {}
        for v in (0, 6, 100):
            for mode in ("clique4_sel", "barbell_sel"):
                ent["%s_%d" % (mode, v)] = O.ref_query_edges(mode, a[:, 0], a[:, 1], value=v)["count_u64"]
        out["facebook_" + key] = ent
    for name in GRAPHS:
        (u, v), sym = _gen(O, name)
        s, d, nn = O.preprocess(u, v, symmetric=sym)
        ent = {}
        for val in values_for(nn):
            for mode in ("clique4_sel", "barbell_sel"):
                ent["%s_%d" % (mode, val)] = O.ref_query_edges(mode, s, d, value=val)["count_u64"]
        out[name] = ent
    golden["select"] = out
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
