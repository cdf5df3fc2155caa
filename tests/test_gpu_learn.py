"""What the trained layout model gains over the density heuristic.

The engine logs per-item device cycles; profiling every set under each
layout is an exhaustive per-set layout search.  The MLP, trained on those
logs by the engine's own kernels, must (1) predict the per-set cost within a
bounded error, (2) pick layouts whose measured cost is closer to the
exhaustive optimum than the heuristic's (lower regret), and (3) change only
speed: the count is the same under the learned layouts."""
import pytest

from emptyheaded_b200 import learn, workloads

pytestmark = pytest.mark.gpu


def test_learned_layouts_beat_heuristic_regret(eh):
    t = workloads.build_rmat_trie(eh, 18, 7)
    want = t.count("triangle")
    model, info = learn.train_from_trie(eh, t, passes=2, epochs=25)
    assert info["median_abs_pct_error"] < 25.0, info
    assert info["regret_learned_pct"] < info["regret_heuristic_pct"], info
    t.relayout(policy=eh.LEARNED, model=model)
    assert t.count("triangle") == want
    h = t.info()
    assert h["n_uinteger"] + h["n_range_bitset"] + h["n_block_bitset"] == h["n_head"]
    t.free()
    model.free()
