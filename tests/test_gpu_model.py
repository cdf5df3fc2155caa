"""The cost model's hand-written fp32 kernels against the oracle's double
restatement (eh_mlp_loss_grad): forward, loss, gradient, SGD.
Tolerance: fp32 accumulation over <= 64 terms, |err| <= 1e-4 + 2e-3*|ref|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ATOL, RTOL = 1e-4, 2e-3


def _data(seed, n, d0, dL):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, d0)).astype(np.float32)
    y = rng.normal(0, 1, (n, dL)).astype(np.float32)
    return x, y


@pytest.mark.parametrize("dims", [[6, 32, 32, 1], [6, 16, 1], [4, 64, 8, 3]])
def test_gradient_matches_oracle(eh, oracle, dims):
    m = eh.Model(dims, seed=5)
    x, y = _data(1, 96, dims[0], dims[-1])
    p = m.params().astype(np.float64)
    loss, g = m.loss_grad(x, y)
    rloss, rg = oracle.mlp_loss_grad(dims, p, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - rloss) <= ATOL + RTOL * abs(rloss)
    np.testing.assert_allclose(g, rg, rtol=RTOL, atol=ATOL)
    m.free()


def test_predict_matches_oracle_forward(eh, oracle):
    dims = [6, 32, 32, 1]
    m = eh.Model(dims, seed=2)
    x, _ = _data(3, 50, 6, 1)
    yhat = m.predict(x)
    # forward via the oracle: loss against zero targets is 0.5*mean(yhat^2)
    p = m.params().astype(np.float64)
    for i in range(0, 50, 7):
        r, _ = oracle.mlp_loss_grad(dims, p, x[i:i + 1].astype(np.float64), np.zeros((1, 1)))
        assert abs(0.5 * float(yhat[i, 0]) ** 2 - r) <= ATOL + RTOL * r


def test_sgd_step_matches_oracle_and_reduces_loss(eh, oracle):
    dims = [6, 16, 1]
    m = eh.Model(dims, seed=9)
    x, y = _data(4, 128, 6, 1)
    p0 = m.params().astype(np.float64)
    _, rg = oracle.mlp_loss_grad(dims, p0, x.astype(np.float64), y.astype(np.float64))
    lr = 0.05
    m.train(x, y, lr=lr, steps=1)
    np.testing.assert_allclose(m.params(), p0 - lr * rg, rtol=RTOL, atol=ATOL)
    l0 = oracle.mlp_loss_grad(dims, p0, x.astype(np.float64), y.astype(np.float64))[0]
    m.train(x, y, lr=lr, steps=200)
    l1 = oracle.mlp_loss_grad(dims, m.params().astype(np.float64), x.astype(np.float64), y.astype(np.float64))[0]
    assert l1 < 0.8 * l0
