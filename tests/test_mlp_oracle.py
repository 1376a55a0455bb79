"""The FP64 surrogate oracle's gradient against central finite differences of its own loss (CPU): the oracle is
pinned by calculus before it checks the GPU."""
import numpy as np

from oracle import mlp_oracle as O

P = 128 * 16 + 128 + 2 * (128 * 128 + 128) + 128 + 1


def test_oracle_gradients_are_the_derivative_of_its_loss():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(P) * 0.1
    sc = np.concatenate([np.zeros(16), np.ones(16), [0.0, 1.0]])
    x = rng.standard_normal((64, 16)).astype(np.float32)
    y = rng.standard_normal(64)
    _, g = O.loss_and_grads(p, sc, x, y, emulate=False)
    idx = np.concatenate([rng.choice(2048, 6, replace=False), 2048 + rng.choice(128, 3, replace=False),
                          2176 + rng.choice(16384, 6, replace=False), 18688 + rng.choice(16384, 6, replace=False),
                          [P - 129, P - 60, P - 1]])
    h = 1e-6
    for i in idx:
        e = np.zeros(P)
        e[i] = h
        lp, _ = O.loss_and_grads(p + e, sc, x, y, emulate=False)
        lm, _ = O.loss_and_grads(p - e, sc, x, y, emulate=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-40], np.float32)
    assert list(O.bf16(x)) == [1.0, 1.0, 1.0078125, -3.140625, np.float32(9.1835496e-41)]
