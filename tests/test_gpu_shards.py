"""The multi-GPU split on one GPU: every rank runs the work items
i % world == rank of the same plan and the partial counts are summed (one
all-reduce across GPUs).  Here the shares run one after another on this GPU
and must sum to the unsharded count, for items cut by probes (density-rule
layouts) and by the cost model's predicted cycles (learned layouts)."""
import pytest

pytestmark = pytest.mark.gpu


def _shares(t, query, world):
    return sum(t.count(query, shard=(r, world)) for r in range(world))


def test_shards_sum_to_the_count(eh, oracle):
    from emptyheaded_b200 import learn, workloads
    t = workloads.build_rmat_trie(eh, 16, 42)
    want = {q: t.count(q) for q in ("triangle", "clique4")}
    for world in (2, 3, 8):
        for q in want:
            assert _shares(t, q, world) == want[q], (q, world)
    model, info, _ = learn.train_from_trie(eh, t, passes=1, epochs=20)
    t.relayout(policy=eh.LEARNED, model=model)
    for world in (2, 3, 8):
        for q in want:
            assert _shares(t, q, world) == want[q], ("learned", q, world)
    t.free()
