"""The MLP oracle's backward pass (float64, no BF16 rounding) against central
finite differences: relative error 1e-6 per tensor."""
import numpy as np

from oracle import mlp_oracle


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [6, 5, 5, 5, 4]
    flat = rng.standard_normal(sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(4))) * 0.5
    n, ntgt = 7, 3
    x = rng.standard_normal((9, dims[0]))
    t = rng.standard_normal((9, dims[4]))

    def loss_of(v):
        return mlp_oracle.loss_and_gradients(mlp_oracle.unflatten(v, dims), x, t, n, ntgt, use_bf16=False)[0]

    _, grads = mlp_oracle.loss_and_gradients(mlp_oracle.unflatten(flat, dims), x, t, n, ntgt, use_bf16=False)
    g = mlp_oracle.flatten(grads)
    h = 1e-6
    fd = np.array([(loss_of(flat + h * e) - loss_of(flat - h * e)) / (2 * h) for e in np.eye(flat.size)])
    assert np.abs(g - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max())


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159265], np.float32)
    r = mlp_oracle.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # halfway, even mantissa kept
    assert r[2] == 1.0078125      # above halfway rounds up
    assert r[3] == 1.0078125
    assert abs(r[4] + 3.140625) < 1e-7
