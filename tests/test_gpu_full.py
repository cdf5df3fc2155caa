"""Full-size checks at the benchmark configuration (R-MAT scale 22, edge
factor 16, a/b/c/d = 0.57/0.19/0.19/0.05, seed 42): the device pipeline
reproduces the exact edge list the reference engine counted (sha1) and the
device count equals the reference's 2,110,948,863 under every layout
policy.  Size-independent properties back it: counts are layout-invariant
and schedule-invariant, and the per-vertex annotation sums to the total."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat22(eh, golden):
    u, v = eh.gen_rmat(42, 22, 16 << 22)
    s, d, nn = eh.preprocess(u, v)
    u.free()
    v.free()
    return s, d, nn, golden["synthetic"]["rmat_s22_ef16_s42"]


def test_rmat22_edge_list_is_the_reference_input(rmat22):
    s, d, nn, g = rmat22
    hs, hd = s.numpy(), d.numpy()
    assert (len(hs), nn) == (g["rows"], g["nodes"])
    assert hashlib.sha1(hs.tobytes() + hd.tobytes()).hexdigest() == g["sha1"]


def test_rmat20_clique4_matches_reference(eh, golden):
    """4-clique configuration: R-MAT scale 20, degree-ordered src < dst;
    the reference engine counts 17,101,670,542."""
    g = golden["synthetic"]["rmat_s20_ef16_s42"]
    u, v = eh.gen_rmat(42, 20, 16 << 20)
    s, d, nn = eh.preprocess(u, v)
    hs, hd = s.numpy(), d.numpy()
    assert hashlib.sha1(hs.tobytes() + hd.tobytes()).hexdigest() == g["sha1"]
    t = eh.Trie(s, d)
    assert t.count("clique4") == g["clique4"] == 17101670542
    t.relayout(policy=2, forced=0, max_bitset_bytes=1 << 50)
    assert t.count("clique4") == g["clique4"]
    t.free()


def test_rmat22_triangle_count_every_layout(eh, rmat22):
    s, d, nn, g = rmat22
    t = eh.Trie(s, d)
    assert t.count("triangle") == g["triangle"] == 2110948863
    for forced in (1, 0, 3):
        # bitsets only where they stay within 16 words per element
        t.relayout(policy=2, forced=forced, max_bitset_bytes=1 << 50)
        assert t.count("triangle") == g["triangle"], forced
    t.relayout()
    ann = t.triangle_annotation()
    assert int(ann.sum(dtype=np.uint64)) == g["triangle"]
    t.free()


def test_chunglu23_lollipop_barbell_match_reference(eh, golden):
    """Barbell / lollipop configuration at full size: Chung-Lu n = 2^23,
    average degree 32, exponent 2.1, symmetrised (221,539,750 rows).  The
    device pipeline gives the edge list the reference engine counted (sha1),
    and the triangle, lollipop and barbell counts equal the reference's;
    the annotation sums to the triangle count (a second code path)."""
    g = golden["synthetic"]["chunglu_n8388608_d32_g2.1_s9_sym"]
    n = 1 << 23
    u, v = eh.gen_chunglu(9, n, n * 16, 2.1)
    s, d, nn = eh.preprocess(u, v, symmetric=True)
    u.free()
    v.free()
    hs, hd = s.numpy(), d.numpy()
    assert (len(hs), nn) == (g["rows"], g["nodes"])
    assert hashlib.sha1(hs.tobytes() + hd.tobytes()).hexdigest() == g["sha1"]
    del hs, hd
    t = eh.Trie(s, d)
    s.free()
    d.free()
    assert t.count("triangle") == g["triangle"]
    assert t.count("lollipop") == g["lollipop"]
    assert t.count("barbell") == g["barbell"]
    assert int(t.triangle_annotation().sum(dtype=np.uint64)) == g["triangle"]
    t.free()
