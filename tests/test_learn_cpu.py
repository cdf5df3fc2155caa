"""Host logic of the learned layout policy that needs no GPU: folding the
feature/target standardisation into the network weights, the feature
vector, and the regret bookkeeping."""
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
