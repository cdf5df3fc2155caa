"""Named synthetic workloads (seeded; no datasets are needed).

rmat(scale)          R-MAT, edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05
batch256()           256 independent R-MAT graphs, scale = round(exp(U(ln 10,
                     ln 18))) from numpy's default_rng(2024), seed 1000 + i
chunglu(n, ...)      Chung-Lu power law, symmetrised (barbell / lollipop)
"""
import numpy as np

ABCD = (0.57, 0.19, 0.19)
EDGE_FACTOR = 16


def batch256_spec(n=256, seed=2024):
    rng = np.random.default_rng(seed)
    scales = np.rint(np.exp(rng.uniform(np.log(10), np.log(18), n))).astype(int)
    return [(int(s), 1000 + i) for i, s in enumerate(scales)]


def build_rmat_trie(E, scale, seed, ctx=None, symmetric=False, **trie_kw):
    """Device pipeline: R-MAT samples -> encoded Edge relation -> trie."""
    u, v = E.gen_rmat(seed, scale, EDGE_FACTOR << scale, *ABCD, ctx=ctx)
    s, d, nodes = E.preprocess(u, v, symmetric=symmetric, ctx=ctx)
    u.free()
    v.free()
    t = E.Trie(s, d, ctx=ctx, **trie_kw)
    s.free()
    d.free()
    return t


def build_chunglu_trie(E, n=1 << 23, avg_degree=32, gamma=2.1, seed=9, ctx=None, **trie_kw):
    """Device pipeline for the barbell / lollipop workload: Chung-Lu power
    law with n nodes and n * avg_degree / 2 undirected samples, symmetrised
    and deduplicated (the reference runs these plans on the duplicated
    relation, test/graph/travis.py:647-692)."""
    u, v = E.gen_chunglu(seed, n, n * avg_degree // 2, gamma, ctx=ctx)
    s, d, nodes = E.preprocess(u, v, symmetric=True, ctx=ctx)
    u.free()
    v.free()
    t = E.Trie(s, d, ctx=ctx, **trie_kw)
    s.free()
    d.free()
    return t


def golden_counts():
    """The reference engine's counts on the seeded workloads
    (tests/golden/golden.json, "synthetic"), for self-checking runs; {} when
    the fixture is absent."""
    import json
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden", "golden.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return json.load(f).get("synthetic", {})
