"""Pins the CPU oracle against the reference: its own golden counts
(test/graph/travis.py), per-pair ops::set_intersect results, trie layouts
and bytes produced by the compiled reference engine (tests/golden)."""
import hashlib

import numpy as np
import pytest

LAYOUT_BITSET = 0


def norm_bitset(raw):
    """Zero the per-word rank of empty words: the reference leaves those
    entries unwritten (range_bitset.hpp:140-151), the fixtures hold zeros."""
    raw = np.array(raw, np.uint8)
    w = (len(raw) - 8) // 12
    words = raw[8: 8 + 8 * w].view(np.uint64)
    rank = raw[8 + 8 * w: 8 + 12 * w].view(np.uint32).copy()
    rank[words == 0] = 0
    return np.concatenate([raw[: 8 + 8 * w], rank.view(np.uint8)])


def test_facebook_goldens(oracle, facebook, golden):
    tr = golden["travis"]
    p = facebook["pruned"]
    t = oracle.Trie(p[:, 0], p[:, 1])
    assert t.triangle() == tr["facebook_pruned"]["triangle"] == 1612010
    assert t.clique4() == tr["facebook_pruned"]["clique4"] == 30004668
    d = facebook["duplicated"]
    t2 = oracle.Trie(d[:, 0], d[:, 1])
    assert t2.lollipop() == tr["facebook_duplicated"]["lollipop"] == 1426911480
    assert t2.barbell() == tr["facebook_duplicated"]["barbell"] == 20371831447136


def test_reference_engine_counts(oracle, facebook, golden):
    """Counts of the compiled reference engine on the in-repo graphs."""
    eng = golden["reference_engine"]
    for name, key in (("facebook_pruned", "pruned"), ("facebook_duplicated", "duplicated"), ("simple", "simple")):
        a = facebook[key]
        t = oracle.Trie(a[:, 0], a[:, 1])
        for mode, want in eng[name].items():
            assert getattr(t, mode)() == want, (name, mode)


SMALL = ["er_16384_131072_s1", "rmat_s12_ef16_s3", "rmat_s14_ef16_s5_sym"]


def _gen(oracle, name):
    if name.startswith("er_"):
        return oracle.gen_er(1, 16384, 131072), False
    if name == "rmat_s12_ef16_s3":
        return oracle.gen_rmat(3, 12, 16 << 12), False
    if name == "rmat_s16_ef16_s42":
        return oracle.gen_rmat(42, 16, 16 << 16), False
    if name == "rmat_s14_ef16_s5_sym":
        return oracle.gen_rmat(5, 14, 16 << 14), True
    if name.startswith("chunglu"):
        return oracle.gen_chunglu(9, 65536, 65536 * 16, 2.1), True
    raise KeyError(name)


@pytest.mark.parametrize("name", SMALL + ["rmat_s16_ef16_s42", "chunglu_n65536_d32_g2.1_s9_sym"])
def test_synthetic_vs_reference_engine(oracle, golden, name):
    """The oracle's generator + preprocessing reproduce the edge lists the
    reference engine counted (sha1), and the oracle's counts equal it."""
    g = golden["synthetic"][name]
    (u, v), sym = _gen(oracle, name)
    s, d, nn = oracle.preprocess(u, v, symmetric=sym)
    assert len(s) == g["rows"] and nn == g["nodes"]
    assert hashlib.sha1(s.tobytes() + d.tobytes()).hexdigest() == g["sha1"]
    t = oracle.Trie(s, d)
    for mode in ("triangle", "clique4", "lollipop", "barbell"):
        if mode in g:
            assert getattr(t, mode)() == g[mode], mode


def test_setops_vs_reference(oracle):
    z = np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "setops.npz"))
    sets = [z["set_elems"][z["set_off"][i]: z["set_off"][i + 1]] for i in range(len(z["set_off"]) - 1)]
    pairs = z["pairs"]
    for p, (a, b) in enumerate(pairs):
        A, B = sets[a], sets[b]
        want = z["elems"][z["elem_off"][p]: z["elem_off"][p + 1]]
        got = oracle.intersect(A, B)
        assert int(z["counts"][p]) == len(got), p
        np.testing.assert_array_equal(got, want)
        # layout decision and the range_bitset bytes of A
        assert oracle.hybrid_type(A) == (int(z["typeA"][p]) if len(A) else 1)
        ab = z["abytes"][z["abytes_off"][p]: z["abytes_off"][p + 1]]
        if len(A) and z["typeA"][p] == LAYOUT_BITSET:
            np.testing.assert_array_equal(norm_bitset(oracle.range_bitset(A)), ab)


@pytest.mark.parametrize("name", ["facebook_pruned", "er", "facebook_duplicated"])
def test_trie_layouts_vs_reference(oracle, facebook, name):
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "triedump.npz"))
    if name == "er":
        u, v = oracle.gen_er(1, 16384, 131072)
        s, d, _ = oracle.preprocess(u, v)
    else:
        a = facebook["pruned" if name == "facebook_pruned" else "duplicated"]
        s, d = a[:, 0], a[:, 1]
    t = oracle.Trie(s, d)
    np.testing.assert_array_equal(t.head, z[name + "_vals"])
    np.testing.assert_array_equal(np.diff(t.off).astype(np.uint32), z[name + "_cards"])
    types = t.layouts()
    np.testing.assert_array_equal(types, z[name + "_types"])
    dig = z[name + "_digests"]
    for i in range(t.n_head):
        c = t.child(i)
        raw = norm_bitset(oracle.range_bitset(c)) if types[i] == LAYOUT_BITSET else np.ascontiguousarray(c, np.uint32).view(np.uint8)
        assert hashlib.sha1(raw.tobytes()).digest() == bytes(dig[i]), i
    # head set
    assert oracle.hybrid_type(t.head) == int(z[name + "_head_type"][0])


def test_mlp_gradient_finite_difference(oracle):
    rng = np.random.default_rng(0)
    dims = [6, 16, 8, 1]
    n = sum(dims[i + 1] * dims[i] + dims[i + 1] for i in range(3))
    p = rng.normal(0, 0.4, n)
    x = rng.normal(0, 1, (32, 6))
    y = rng.normal(0, 1, (32, 1))
    loss, g = oracle.mlp_loss_grad(dims, p, x, y)
    eps = 1e-6
    for k in rng.choice(n, 40, replace=False):
        q = p.copy()
        q[k] += eps
        lp, _ = oracle.mlp_loss_grad(dims, q, x, y)
        q[k] -= 2 * eps
        lm, _ = oracle.mlp_loss_grad(dims, q, x, y)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_triangle_listing_goldens(oracle, facebook):
    """Triangle(a,b,c) and TriangleProj(a,b) on facebook_pruned:
    1612010 rows with row0 (6,5,2), 85658 rows with row0 (6,5)
    (test/graph/travis.py:282-318)."""
    p = facebook["pruned"]
    t = oracle.Trie(p[:, 0], p[:, 1])
    rows = t.triangle_tuples()
    assert len(rows) == 1612010 and tuple(rows[0]) == (6, 5, 2)
    proj = t.triangle_projection()
    assert len(proj) == 85658 and tuple(proj[0]) == (6, 5)
    # the projected attribute c is not intersected by the reference plan:
    # more rows than the pairs that close a triangle
    assert len(np.unique(rows[:, :2], axis=0)) == 84185


def test_selection_goldens(oracle, facebook, golden):
    """FliqueSelAgg x=0 -> 3759972 and BarbellSelAgg p=6 -> 26936100 on
    facebook_duplicated (test/graph/travis.py:385-401, 472-487)."""
    tr = golden["travis"]["facebook_duplicated"]
    d = facebook["duplicated"]
    t = oracle.Trie(d[:, 0], d[:, 1])
    assert t.clique4_sel(0) == tr["clique4_sel_x0"] == 3759972
    assert t.barbell_sel(6) == tr["barbell_sel_p6"] == 26936100


@pytest.mark.parametrize("name", ["facebook_duplicated", "facebook_pruned"] + SMALL)
def test_selection_vs_reference_engine(oracle, facebook, golden, name):
    """Selection counts of the compiled reference engine (its selection
    bags, several selected values per graph) equal the oracle's."""
    if name.startswith("facebook"):
        a = facebook[name.split("_")[1]]
        s, d = a[:, 0], a[:, 1]
    else:
        (u, v), sym = _gen(oracle, name)
        s, d, _ = oracle.preprocess(u, v, symmetric=sym)
    t = oracle.Trie(s, d)
    for key, want in golden["select"][name].items():
        mode, val = key.rsplit("_", 1)
        assert getattr(t, mode)(int(val)) == want, key


def test_encoding_vs_reference(oracle):
    """The numpy restatement of Encoding<T> equals the reference's own
    Encoding<T> (fixture from oracle/_ref/eh_ref encode) for every numeric
    value type: key_to_value table (bit for bit) and every key."""
    z = np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "encoding.npz"))
    for vt in oracle.VALUE_TYPES:
        cols = [z["%s_col%d" % (vt, j)] for j in range(3)]
        values, keys = oracle.encoding(cols, vt)
        assert values.tobytes() == z[vt + "_values"].tobytes(), vt
        for j, k in enumerate(keys):
            np.testing.assert_array_equal(k, z["%s_keys%d" % (vt, j)])


def _refdb_dirs(tmp, names=None):
    z = np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "refdb.npz"))
    os = __import__("os")
    out = {}
    for key in z.files:
        name, fn = key.split("/")
        if fn == "threads" or (names and name not in names):
            continue
        ram = os.path.join(str(tmp), name, "ram")
        os.makedirs(ram, exist_ok=True)
        with open(os.path.join(ram, fn), "wb") as f:
            f.write(z[key].tobytes())
        out[name] = (os.path.join(str(tmp), name), int(z[name + "/threads"][0]))
    return out


def test_reference_trie_files(oracle, facebook, tmp_path):
    """The restatement of the on-disk format reads the tries the reference
    saved (fixture) into the same CSR the oracle builds from the edges, and
    what it writes the reference engine loads (triangle count unchanged)."""
    dirs = _refdb_dirs(tmp_path)
    p = facebook["pruned"]
    want = {"facebook_pruned": (p[:, 0], p[:, 1])}
    for name in ("rmat_s12_ef16_s3", "rmat_s14_ef16_s5_sym"):
        (u, v), sym = _gen(oracle, name)
        s, d, _ = oracle.preprocess(u, v, symmetric=sym)
        want[name] = (s, d)
    for name, (path, thr) in dirs.items():
        t = oracle.Trie(*want[name])
        head, off, vals, types = oracle.read_reference_trie(path)
        np.testing.assert_array_equal(head, t.head)
        np.testing.assert_array_equal(off, t.off)
        np.testing.assert_array_equal(vals, t.vals)
        np.testing.assert_array_equal(types[:-1], t.layouts())
        if oracle.ref_available():
            out = str(tmp_path / ("w_" + name))
            oracle.write_reference_trie(out, t.head, t.off, t.vals, len(t.vals), thr + 1)
            assert oracle.ref_load_triangle(out, thr + 1)["count_u64"] == t.triangle(), name
