"""Parity of the sm_100a path (through the C ABI) with the oracle and the
reference's golden vectors.  Integer work: every comparison is exact."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

UINT, BITSET, BLOCK = 1, 0, 3
POLICIES = [("heuristic", 0, 1), ("uint", 2, UINT), ("bitset", 2, BITSET), ("block", 2, BLOCK)]


def norm_bitset(raw):
    raw = np.array(raw, np.uint8)
    w = (len(raw) - 8) // 12
    words = raw[8: 8 + 8 * w].view(np.uint64)
    rank = raw[8 + 8 * w: 8 + 12 * w].view(np.uint32).copy()
    rank[words == 0] = 0
    return np.concatenate([raw[: 8 + 8 * w], rank.view(np.uint8)])


# ----------------------------------------------------------- input pipeline
def test_generators_match_oracle(eh, oracle, ctx):
    u, v = eh.gen_er(1, 16384, 131072)
    ou, ov = oracle.gen_er(1, 16384, 131072)
    np.testing.assert_array_equal(u.numpy(), ou)
    np.testing.assert_array_equal(v.numpy(), ov)
    u, v = eh.gen_rmat(3, 12, 16 << 12)
    ou, ov = oracle.gen_rmat(3, 12, 16 << 12)
    np.testing.assert_array_equal(u.numpy(), ou)
    np.testing.assert_array_equal(v.numpy(), ov)
    u, v = eh.gen_chunglu(9, 65536, 65536 * 16, 2.1)
    ou, ov = oracle.gen_chunglu(9, 65536, 65536 * 16, 2.1)
    np.testing.assert_array_equal(u.numpy(), ou)
    np.testing.assert_array_equal(v.numpy(), ov)


@pytest.mark.parametrize("name,gen,sym", [
    ("er_16384_131072_s1", lambda E: E.gen_er(1, 16384, 131072), False),
    ("rmat_s12_ef16_s3", lambda E: E.gen_rmat(3, 12, 16 << 12), False),
    ("rmat_s16_ef16_s42", lambda E: E.gen_rmat(42, 16, 16 << 16), False),
    ("rmat_s14_ef16_s5_sym", lambda E: E.gen_rmat(5, 14, 16 << 14), True),
    ("chunglu_n65536_d32_g2.1_s9_sym", lambda E: E.gen_chunglu(9, 65536, 65536 * 16, 2.1), True),
])
def test_preprocess_and_counts_vs_reference_engine(eh, golden, name, gen, sym):
    """Device generator + preprocessing give the exact edge list the
    reference engine counted; device counts equal the reference's under
    every layout policy."""
    g = golden["synthetic"][name]
    u, v = gen(eh)
    s, d, nn = eh.preprocess(u, v, symmetric=sym)
    hs, hd = s.numpy(), d.numpy()
    assert (len(hs), nn) == (g["rows"], g["nodes"])
    assert hashlib.sha1(hs.tobytes() + hd.tobytes()).hexdigest() == g["sha1"]
    for _, policy, forced in POLICIES:
        t = eh.Trie(s, d, policy=policy, forced=forced)
        for mode in ("triangle", "clique4", "lollipop", "barbell"):
            if mode in g:
                assert t.count(mode) == g[mode], (name, mode, policy, forced)
        t.free()


# --------------------------------------------------------------------- trie
@pytest.mark.parametrize("name", ["facebook_pruned", "facebook_duplicated", "er"])
def test_trie_matches_reference_dump(eh, oracle, facebook, name):
    z = np.load(os.path.join(GOLDEN, "triedump.npz"))
    if name == "er":
        u, v = oracle.gen_er(1, 16384, 131072)
        s, d, _ = oracle.preprocess(u, v)
    else:
        a = facebook["pruned" if name == "facebook_pruned" else "duplicated"]
        s, d = a[:, 0], a[:, 1]
    # rows shuffled and duplicated: the build must sort and dedup
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.permutation(len(s)), rng.choice(len(s), len(s) // 7)])
    t = eh.Trie(s[idx], d[idx])
    head, off, vals, lay = t.export()
    np.testing.assert_array_equal(head, z[name + "_vals"])
    np.testing.assert_array_equal(np.diff(off).astype(np.uint32), z[name + "_cards"])
    np.testing.assert_array_equal(lay, z[name + "_types"])
    o = oracle.Trie(s, d)
    np.testing.assert_array_equal(vals, o.vals)
    dig = z[name + "_digests"]
    for i in range(len(head)):
        raw, l = t.set_bytes(i)
        assert l == z[name + "_types"][i]
        if l == BITSET:
            raw = norm_bitset(raw)
        assert hashlib.sha1(raw.tobytes()).digest() == bytes(dig[i]), i
    raw, l = t.set_bytes(None)
    assert l == z[name + "_head_type"][0]
    if l == BITSET:
        raw = norm_bitset(raw)
    assert hashlib.sha1(raw.tobytes()).digest() == bytes(z[name + "_head_digest"])


def test_forced_layout_bytes(eh, oracle):
    u, v = oracle.gen_rmat(3, 12, 16 << 12)
    s, d, _ = oracle.preprocess(u, v)
    o = oracle.Trie(s, d)
    for forced in (BITSET, BLOCK, UINT):
        t = eh.Trie(s, d, policy=2, forced=forced)
        for i in range(0, o.n_head, 7):
            raw, l = t.set_bytes(i)
            assert l == forced
            c = o.child(i)
            want = {BITSET: oracle.range_bitset(c), BLOCK: oracle.block_bitset(c),
                    UINT: np.ascontiguousarray(c, np.uint32).view(np.uint8)}[forced]
            np.testing.assert_array_equal(raw, want)
        t.free()


def test_trie_edge_cases(eh):
    t = eh.Trie(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert t.info()["n_head"] == 0 and t.count("triangle") == 0
    t = eh.Trie(np.array([3], np.uint32), np.array([7], np.uint32))
    head, off, vals, lay = t.export()
    assert list(head) == [3] and list(vals) == [7] and t.count("triangle") == 0
    # a single triangle, both directions, self-loop and duplicates
    s = np.array([0, 0, 1, 1, 1, 2, 0], np.uint32)
    d = np.array([1, 2, 2, 2, 1, 0, 1], np.uint32)
    t = eh.Trie(s, d)
    head, off, vals, _ = t.export()
    assert list(head) == [0, 1, 2] and list(vals) == [1, 2, 1, 2, 0]


# ------------------------------------------------------------------ set ops
@pytest.mark.parametrize("assign", ["heuristic", "uint", "bitset", "block", "mixed"])
def test_set_intersect_vs_reference(eh, oracle, assign):
    z = np.load(os.path.join(GOLDEN, "setops.npz"))
    off = z["set_off"]
    sets = [z["set_elems"][off[i]: off[i + 1]] for i in range(len(off) - 1)]
    pairs = z["pairs"]
    if assign == "heuristic":
        lay = [oracle.hybrid_type(s) if len(s) else UINT for s in sets]
    elif assign == "mixed":
        rng = np.random.default_rng(3)
        lay = rng.choice([UINT, BITSET, BLOCK], len(sets))
    else:
        lay = [{"uint": UINT, "bitset": BITSET, "block": BLOCK}[assign]] * len(sets)
    counts, mats = eh.set_intersect(sets, lay, pairs, materialize=True)
    np.testing.assert_array_equal(counts, z["counts"])
    for p in range(len(pairs)):
        np.testing.assert_array_equal(mats[p], z["elems"][z["elem_off"][p]: z["elem_off"][p + 1]])
    assert np.array_equal(eh.set_intersect(sets, lay, pairs), counts)


def test_set_intersect_rejects_unsorted(eh):
    with pytest.raises(eh.EHError):
        eh.set_intersect([np.array([3, 1], np.uint32), np.array([1], np.uint32)], [UINT, UINT], [[0, 1]])


# ------------------------------------------------------------------ queries
@pytest.mark.parametrize("label,policy,forced", POLICIES)
def test_facebook_goldens_on_device(eh, facebook, golden, label, policy, forced):
    tr = golden["travis"]
    p = facebook["pruned"]
    t = eh.Trie(p[:, 0], p[:, 1], policy=policy, forced=forced)
    assert t.count("triangle") == tr["facebook_pruned"]["triangle"] == 1612010
    assert t.count("clique4") == tr["facebook_pruned"]["clique4"] == 30004668
    d = facebook["duplicated"]
    t2 = eh.Trie(d[:, 0], d[:, 1], policy=policy, forced=forced)
    assert t2.count("lollipop") == tr["facebook_duplicated"]["lollipop"] == 1426911480
    assert t2.count("barbell") == tr["facebook_duplicated"]["barbell"] == 20371831447136
    eng = golden["reference_engine"]
    for m, want in eng["facebook_duplicated"].items():
        if m in eh.QUERIES:  # path2 has no named plan (the C++ layer's host loop runs it)
            assert t2.count(m) == want, m
    s = facebook["simple"]
    t3 = eh.Trie(s[:, 0], s[:, 1], policy=policy, forced=forced)
    for m, want in eng["simple"].items():
        if m in eh.QUERIES:
            assert t3.count(m) == want, m


def test_general_direction_relation(eh, oracle):
    """A directed relation with cycles and some mirrored rows: neither up,
    down nor symmetric; the device must still equal the generic loop nest."""
    rng = np.random.default_rng(11)
    s = rng.integers(0, 300, 6000).astype(np.uint32)
    d = rng.integers(0, 300, 6000).astype(np.uint32)
    o = oracle.Trie(s, d)
    for _, policy, forced in POLICIES:
        t = eh.Trie(s, d, policy=policy, forced=forced)
        assert t.count("triangle") == o.triangle()
        assert t.count("clique4") == o.clique4()
        assert t.count("lollipop") == o.lollipop()
        assert t.count("barbell") == o.barbell()
        np.testing.assert_array_equal(t.triangle_annotation(), o.triangle_per_vertex())


def test_annotation_symmetric(eh, oracle, facebook):
    d = facebook["duplicated"]
    t = eh.Trie(d[:, 0], d[:, 1])
    o = oracle.Trie(d[:, 0], d[:, 1])
    np.testing.assert_array_equal(t.triangle_annotation(), o.triangle_per_vertex())


def test_schedule_knobs_do_not_change_counts(eh, oracle):
    u, v = oracle.gen_rmat(42, 16, 16 << 16)
    s, d, _ = oracle.preprocess(u, v)
    want = 15754143
    t = eh.Trie(s, d)
    for warps in (1, 4, 8, 16):
        for chunk in (1, 64, 4096, 1 << 22):
            for smem in (64, 2048, 8192):
                assert t.count("triangle", warps=warps, chunk=chunk, smem_words=smem) == want
    for long_row in (1, 7, 32, 1 << 20):
        assert t.count("triangle", long_row=long_row) == want
    t.relayout(policy=2, forced=0, max_bitset_bytes=1 << 50)
    for long_row in (1, 32, 1 << 20):
        for smem in (64, 1024):
            assert t.count("triangle", long_row=long_row, smem_words=smem) == want


def test_batched_counts(eh, oracle):
    tries, want = [], []
    for k, sc in enumerate((8, 10, 11, 12, 9, 13)):
        u, v = oracle.gen_rmat(100 + k, sc, 16 << sc)
        s, d, _ = oracle.preprocess(u, v)
        tries.append(eh.Trie(s, d))
        want.append(oracle.Trie(s, d).triangle())
    got = eh.count_batched(tries)
    np.testing.assert_array_equal(got, np.array(want, np.uint64))
    got4 = eh.count_batched(tries, "clique4")
    np.testing.assert_array_equal(got4, np.array([t.count("clique4") for t in tries], np.uint64))


def test_host_csr_entry(eh, oracle, golden):
    u, v = oracle.gen_rmat(3, 12, 16 << 12)
    s, d, nn = oracle.preprocess(u, v)
    o = oracle.Trie(s, d)
    r = eh.count_host_csr(o.head, o.off, o.vals, nn)
    assert r == golden["synthetic"]["rmat_s12_ef16_s3"]["triangle"]


@pytest.mark.parametrize("kind", ["up", "symmetric", "general", "hint_too_small", "big_up"])
def test_host_csr_overlapped_build(eh, oracle, facebook, golden, kind):
    """The host-buffer entry copies the values in chunks while it computes the
    reverse level's keys as if every row went up; relations that do not go up,
    and values beyond the caller's value-domain hint, take the regular build.
    Every count must equal the oracle's."""
    if kind == "symmetric":
        a = facebook["duplicated"]
        s, d = a[:, 0], a[:, 1]
    elif kind == "general":
        rng = np.random.default_rng(5)
        s = rng.integers(0, 400, 8000).astype(np.uint32)
        d = rng.integers(0, 400, 8000).astype(np.uint32)
    elif kind == "big_up":
        u, v = oracle.gen_rmat(42, 18, 16 << 18)
        s, d, _ = oracle.preprocess(u, v)
    else:
        u, v = oracle.gen_rmat(3, 12, 16 << 12)
        s, d, _ = oracle.preprocess(u, v)
    o = oracle.Trie(s, d)
    hint = 1 if kind == "hint_too_small" else int(max(s.max(), d.max())) + 1
    for q in ("triangle", "clique4", "lollipop"):
        got = eh.count_host_csr(o.head, o.off, o.vals, hint, query=q)
        assert got == getattr(o, q)(), (kind, q)


def test_autotune_keeps_counts(eh, oracle):
    from emptyheaded_b200 import autotune
    u, v = oracle.gen_rmat(42, 16, 16 << 16)
    s, d, _ = oracle.preprocess(u, v)
    t = eh.Trie(s, d)
    grid = {"smem_words": (512, 1024), "chunk": (4096, 32768), "long_row": (16, 64), "warps": (4, 8)}
    best, log = autotune.tune(t, reps=1, rounds=1, grid=grid)
    assert set(best) == set(autotune.DEFAULT) and len(log) >= 5
    assert t.count("triangle", config=best) == 15754143


def test_context_close_frees_dependents(eh, facebook):
    """Closing a context first frees the tries and models made in it, so
    no handle outlives its context (interpreter exit relies on this)."""
    c = eh.Context(0)
    p = facebook["pruned"]
    t = eh.Trie(p[:, 0], p[:, 1], ctx=c)
    m = eh.Model([6, 8, 1], ctx=c)
    assert t.count("triangle") == 1612010
    c.close()
    assert t.h is None and m.h is None
    t.free()
    c.close()


@pytest.mark.parametrize("smem", [64, 256, 1024])
def test_compressed_bitset_staging(eh, oracle, smem):
    """Range bitsets too large for a warp's region are staged compressed
    (presence bits, ranks, non-zero words) when that fits: forcing every
    admissible set to a bitset and shrinking the region sends most sets
    through that path, in the COUNT, 4-clique, annotated and materializing
    kernels.  Counts and rows must not change."""
    u, v = oracle.gen_rmat(42, 14, 16 << 14)
    s, d, _ = oracle.preprocess(u, v)
    o = oracle.Trie(s, d)
    t = eh.Trie(s, d, policy=2, forced=0, max_bitset_bytes=1 << 50)
    cfg = {"smem_words": smem}
    assert t.count("triangle", config=cfg) == o.triangle()
    assert t.count("clique4", config=cfg) == o.clique4()
    assert t.count("lollipop", config=cfg) == o.lollipop()
    assert t.count("barbell", config=cfg) == o.barbell()
    assert t.count("triangle", config=dict(cfg, warps=4, long_row=1)) == o.triangle()
    t.free()
    a = oracle.Trie(*(np.array(x, np.uint32) for x in (s, d)))
    ts = eh.Trie(s, d, policy=2, forced=0, max_bitset_bytes=1 << 50)
    np.testing.assert_array_equal(ts.materialize(), a.triangle_tuples())
    ts.free()
