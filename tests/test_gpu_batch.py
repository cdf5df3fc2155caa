"""The batched configuration: 256 independent seeded R-MAT graphs (scales
log-uniform in 10..18), one persistent kernel over every graph's work
items, captured once as a CUDA graph and replayed.  Each graph's count must
equal the reference engine's (tests/golden/golden.json "batch256")."""
import numpy as np
import pytest

from emptyheaded_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_tries(eh):
    tries = [workloads.build_rmat_trie(eh, sc, sd) for sc, sd in workloads.batch256_spec()]
    yield tries
    for t in tries:
        t.free()


def test_batch256_matches_reference(eh, golden, batch_tries):
    want = np.array([g["triangle"] for g in golden["batch256"]], np.uint64)
    b = eh.Batch(batch_tries)
    got, st = b.run(stats=True)
    np.testing.assert_array_equal(got, want)
    assert st["launches"] == 1
    np.testing.assert_array_equal(b.run(), want)  # replay
    b.free()
    # the per-trie path agrees on a sample
    for t, w in list(zip(batch_tries, want))[::37]:
        assert t.count("triangle") == w


def test_batch_clique4_matches_per_trie(eh, batch_tries):
    small = [t for t in batch_tries if t.info()["rows"] < 200000][:12]
    b = eh.Batch(small, "clique4")
    np.testing.assert_array_equal(b.run(), np.array([t.count("clique4") for t in small], np.uint64))
    b.free()
