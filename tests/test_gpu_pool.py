"""The engine's device memory pool: eh_context_memory reports what it holds
and uses, eh_context_reserve keeps one block that later calls are carved
from.  A host-CSR COUNT whose peak fits the reserved block maps no new
memory, and what it used returns to the pool (the count itself is checked
against the facebook_pruned triangle golden)."""
import pytest

pytestmark = pytest.mark.gpu


def test_reserve_and_reuse(eh, ctx, facebook, golden):
    p = facebook["pruned"]
    t = eh.Trie(p[:, 0], p[:, 1], ctx=ctx)
    head, off, vals, _ = t.export()
    n = t.info()["n_nodes"]
    t.free()

    ctx.reserve(0)
    m0 = ctx.memory()
    assert m0["peak"] == m0["used"]
    assert m0["reserved"] >= m0["used"]
    assert eh.count_host_csr(head, off, vals, n, ctx=ctx) == golden["travis"]["facebook_pruned"]["triangle"]
    m1 = ctx.memory()
    assert m1["used"] == m0["used"]  # every buffer of the call went back
    need = m1["peak"] - m0["used"]
    assert need > vals.nbytes  # the call held at least its own copy of the rows

    ctx.reserve(2 * need)
    m2 = ctx.memory()
    assert m2["reserved"] >= m2["used"] + 2 * need
    assert m2["peak"] == m2["used"]
    for _ in range(3):
        assert eh.count_host_csr(head, off, vals, n, ctx=ctx) == golden["travis"]["facebook_pruned"]["triangle"]
    m3 = ctx.memory()
    assert m3["reserved"] == m2["reserved"]  # the calls fit: the pool did not grow
    assert m3["used"] == m2["used"]
    assert m2["used"] < m3["peak"] <= m2["used"] + 2 * need


def test_reserve_zero_trims(eh, ctx):
    ctx.reserve(64 << 20)
    assert ctx.memory()["reserved"] >= 64 << 20
    ctx.reserve(0)
    m = ctx.memory()
    # only blocks still in use stay (allocation granularity aside)
    assert m["reserved"] - m["used"] < 64 << 20
