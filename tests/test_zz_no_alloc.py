"""eh_query_count_noalloc: the COUNT query for callers that must not
allocate device memory while they query (an embedding host whose device
memory belongs to another allocator).  Its scratch is one fixed 64 MiB
device array inside the library instead of per-call allocations.

Checked through the C ABI against eh_query_count (the allocating entry) and
against the reference engine's own counts (tests/golden/golden.json) on two
calls in a row: integer counts, so the comparison is exact.  Collected last
on purpose, and written to pass alone in a fresh process as well."""
import ctypes
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRIANGLE, CLIQUE4 = 0, 1


def _noalloc(eh, ctx, trie, query):
    r = ctypes.c_uint64()
    st = eh.lib().eh_query_count_noalloc(ctx.h, trie.h, query, None, ctypes.byref(r))
    return st, r.value


def _allocating(eh, ctx, trie, query):
    r = ctypes.c_uint64()
    assert eh.lib().eh_query_count(ctx.h, trie.h, query, None, ctypes.byref(r), None) == 0
    return r.value


@pytest.fixture(scope="module")
def nctx(eh):
    return eh.default_context()


@pytest.mark.parametrize("which", ["pruned", "duplicated"])
def test_noalloc_matches_allocating_entry_facebook(eh, nctx, facebook, which):
    a = facebook[which]
    t = eh.Trie(a[:, 0], a[:, 1], ctx=nctx)
    want = _allocating(eh, nctx, t, TRIANGLE)
    for _ in range(2):  # two calls in a row: the array keeps the last call's contents
        st, got = _noalloc(eh, nctx, t, TRIANGLE)
        assert st == 0, eh.lib().eh_last_error()
        assert got == want
    if which == "pruned":
        assert want == 1612010
    t.free()


def _golden(key):
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")) as f:
        return json.load(f)["synthetic"][key]


@pytest.mark.parametrize("case", [(42, 16, False, "rmat_s16_ef16_s42"), (5, 14, True, "rmat_s14_ef16_s5_sym")])
def test_noalloc_matches_reference_counts_rmat(eh, nctx, oracle, case):
    """R-MAT-16 (up-oriented) and a symmetric R-MAT-14, whose largest set
    (3,544 elements) is too large to stage in shared memory for the
    4-clique: its per-warp S buffers then come out of the fixed array."""
    seed, scale, sym, key = case
    g = _golden(key)
    u, v = oracle.gen_rmat(seed, scale, 16 << scale)
    s, d, _ = oracle.preprocess(u, v, symmetric=sym)
    t = eh.Trie(s, d, ctx=nctx)
    for q, name in ((TRIANGLE, "triangle"), (CLIQUE4, "clique4")):
        want = _allocating(eh, nctx, t, q)
        assert want == g[name]
        for _ in range(2):
            st, got = _noalloc(eh, nctx, t, q)
            assert st == 0, eh.lib().eh_last_error()
            assert got == want == g[name]
    t.free()


def test_noalloc_rejects_a_trie_over_its_limit(eh, nctx):
    """9M head entries need more than the 64 MiB array holds: a clear
    EH_ERR_UNSUPPORTED, and the next call still works."""
    n = 9_000_000
    src = np.arange(n, dtype=np.uint32)
    t = eh.Trie(src, src + 1, ctx=nctx)
    st, _ = _noalloc(eh, nctx, t, TRIANGLE)
    assert st == 5  # EH_ERR_UNSUPPORTED
    assert b"allocation-free" in eh.lib().eh_last_error()
    t.free()
    small = eh.Trie(np.array([0, 0, 1], np.uint32), np.array([1, 2, 2], np.uint32), ctx=nctx)
    st, got = _noalloc(eh, nctx, small, TRIANGLE)
    assert st == 0 and got == 1
    small.free()


def test_noalloc_rejects_a_clique_set_over_its_limit(eh, nctx):
    """A 4-clique whose largest set needs per-warp S buffers beyond what the
    64 MiB array has left (a star of 2.2M leaves: 8 warps x 2.2M x 4 bytes
    per block): a clear EH_ERR_UNSUPPORTED naming the largest set, and the
    next call still works."""
    n = 2_200_000
    leaves = np.arange(1, n + 1, dtype=np.uint32)
    t = eh.Trie(np.zeros(n, np.uint32), leaves, ctx=nctx)
    st, _ = _noalloc(eh, nctx, t, CLIQUE4)
    assert st == 5  # EH_ERR_UNSUPPORTED
    assert b"largest set" in eh.lib().eh_last_error()
    st, got = _noalloc(eh, nctx, t, TRIANGLE)
    assert st == 0 and got == 0
    t.free()
