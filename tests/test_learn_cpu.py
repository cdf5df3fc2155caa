"""Host logic of the learned layout policy that needs no GPU: folding the
feature/target standardisation into the network weights, the feature
vector, the exhaustive search's assignment, the training rows (cost-weighted,
capped), pooled profiles, and the regret bookkeeping with the chooser's
margin."""
import numpy as np

from emptyheaded_b200 import learn


def _forward(params, dims, x):
    o, a = 0, x.astype(np.float64)
    for l in range(len(dims) - 1):
        din, dout = dims[l], dims[l + 1]
        W = params[o: o + din * dout].reshape(dout, din)
        b = params[o + din * dout: o + din * dout + dout]
        o += din * dout + dout
        a = a @ W.T + b
        if l + 1 < len(dims) - 1:
            a = np.maximum(a, 0)
    return a


def test_fold_matches_standardised_network():
    rng = np.random.default_rng(0)
    dims = learn.DIMS
    n = sum(dims[i + 1] * dims[i] + dims[i + 1] for i in range(len(dims) - 1))
    p = rng.normal(0, 0.3, n).astype(np.float32)
    x = rng.normal(3, 2, (50, dims[0]))
    mu_x, sd_x = x.mean(0), x.std(0)
    mu_y, sd_y = 12.5, 3.0
    want = _forward(p.astype(np.float64), dims, (x - mu_x) / sd_x) * sd_y + mu_y
    got = _forward(learn._fold(p, dims, mu_x, sd_x, mu_y, sd_y).astype(np.float64), dims, x)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-3)


def test_feature_vector():
    f = learn.set_features(np.array([4.0]), np.array([63.0]), np.array([100.0]), np.array([learn.BITSET]))
    assert f.shape == (1, 6)
    np.testing.assert_allclose(f[0], [np.log1p(4), np.log1p(63), 4 / 64, np.log1p(100), 1, 0], rtol=1e-6)


def _profile(n=6):
    """A synthetic profile: per-set cycles under each layout (NaN: not
    admissible), the density rule's layout, and probe counts."""
    nan = np.nan
    cyc = {
        learn.UINT: np.array([100.0, 400.0, 50.0, 30.0, 900.0, 0.0][:n]),
        learn.BITSET: np.array([80.0, 100.0, nan, 29.0, 1000.0, 0.0][:n]),
        learn.BLOCK: np.array([120.0, 390.0, 60.0, 40.0, 880.0, 0.0][:n]),
    }
    return dict(lens=np.array([10.0, 20, 30, 40, 50, 60])[:n], range=np.array([1e3, 2e3, 3e3, 4e3, 5e3, 6e3])[:n],
                pairs=np.array([5.0, 6, 7, 8, 9, 0])[:n], cycles=cyc,
                heuristic=np.array([learn.UINT, learn.UINT, learn.UINT, learn.BITSET, learn.UINT, learn.UINT])[:n],
                words=np.array([16.0, 32, 47, 63, 79, 94])[:n])


def test_best_layouts_picks_cheapest_admissible_and_keeps_rule_for_unstaged():
    prof = _profile()
    best = learn.best_layouts(prof)
    assert list(best[:5]) == [learn.BITSET, learn.BITSET, learn.UINT, learn.BITSET, learn.BLOCK]
    assert best[5] == learn.UINT  # never probed: the density rule's layout


def test_dataset_oversamples_costly_sets_and_caps_rows():
    prof = _profile()
    x, y = learn.dataset(prof, max_weight=32, max_rows=0)
    staged = prof["pairs"] > 0
    # one row per staged set and admissible layout, repeated by cost / mean cost (1..32)
    want = 0
    for L in learn.LAYOUTS:
        c = prof["cycles"][L]
        m = staged & np.isfinite(c) & (c > 0)
        want += int(np.clip(np.round(c[m] / c[m].mean()), 1, 32).sum())
    assert len(x) == len(y) == want
    assert np.isclose(y.max(), np.log1p(1000.0))
    xc, yc = learn.dataset(prof, max_weight=32, max_rows=7, seed=3)
    assert len(xc) == len(yc) == 7
    # the capped rows are rows of the full set
    full = {tuple(np.round(r, 5)) + (round(float(v), 5),) for r, v in zip(x, y[:, 0])}
    assert all(tuple(np.round(r, 5)) + (round(float(v), 5),) in full for r, v in zip(xc, yc[:, 0]))


def test_merge_profiles_concatenates_sets():
    a, b = _profile(6), _profile(4)
    m = learn.merge_profiles([a, b])
    assert len(m["lens"]) == 10
    for L in learn.LAYOUTS:
        np.testing.assert_array_equal(m["cycles"][L], np.concatenate([a["cycles"][L], b["cycles"][L]]))
    np.testing.assert_array_equal(m["heuristic"], np.concatenate([a["heuristic"], b["heuristic"]]))


class _FakeModel:
    """Predicts log1p(cycles) from a table keyed by (set, layout one-hot)."""

    def __init__(self, prof, factor):
        self.prof, self.factor = prof, factor

    def predict(self, f):
        n = len(f)
        lay = np.where(f[:, 4] > 0.5, learn.BITSET, np.where(f[:, 5] > 0.5, learn.BLOCK, learn.UINT))
        out = np.empty((n, 1), np.float32)
        for i in range(n):
            c = self.prof["cycles"][int(lay[i])][i]
            c = 1e6 if not np.isfinite(c) else c
            out[i, 0] = np.log1p(c * self.factor.get((i, int(lay[i])), 1.0))
        return out


def test_evaluate_applies_the_choosers_margin():
    prof = _profile()
    exact = learn.evaluate(None, _FakeModel(prof, {}), prof, min_gain=0.0)
    assert exact["regret_learned_pct"] < 1e-9  # exact predictions, no margin: the exhaustive optimum
    kept = learn.evaluate(None, _FakeModel(prof, {}), prof, min_gain=0.1)
    # sets 0 (uint 100 -> bitset 80, a 20% gain) and 1 (400 -> bitset 100) move;
    # set 4 (uint 900 -> block 880, a 2% gain) keeps the rule's layout
    best_total = 80 + 100 + 50 + 29 + 880
    chosen_total = 80 + 100 + 50 + 29 + 900
    assert np.isclose(kept["regret_learned_pct"], (chosen_total / best_total - 1) * 100)
    rule_total = 100 + 400 + 50 + 29 + 900
    assert np.isclose(kept["regret_heuristic_pct"], (rule_total / best_total - 1) * 100)
