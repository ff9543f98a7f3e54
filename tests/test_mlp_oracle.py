"""The FP64 MLP reference (oracle/mlp.py) is pinned by central finite
differences of its own loss (no GPU)."""
import numpy as np

from oracle import mlp as M


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n = 6
    layers = []
    for i, o in M.DIMS:
        layers.append((rng.uniform(-1, 1, (o, i)) * np.sqrt(3.0 / i), rng.uniform(-0.1, 0.1, o)))
    flat = M.flatten(layers)
    x = rng.uniform(0, 1, (n, 65))
    y = rng.normal(size=(n, 5))
    loss, g = M.loss_and_grads(flat, x, y)
    idx = rng.choice(flat.size, 40, replace=False)
    # include the first layer's weights and the last layer's bias
    idx = np.concatenate([idx, [0, 65 * 256 + 3, flat.size - 1]])
    h = 1e-6
    for k in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[k] += h
        fm[k] -= h
        num = (M.loss_and_grads(fp, x, y)[0] - M.loss_and_grads(fm, x, y)[0]) / (2 * h)
        assert abs(num - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-8, (k, num, g[k])
    assert loss > 0
