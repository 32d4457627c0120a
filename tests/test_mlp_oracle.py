"""CPU checks of the network oracle (oracle/mlp_oracle.py) that checks the
GPU training kernels: its backward pass against finite differences, and its
BF16 rounding against the IEEE definition."""
import numpy as np

from oracle import mlp_oracle as mo


def _params(rng):
    W1 = rng.normal(0, 0.5, (128, 8))
    W2 = rng.normal(0, 0.1, (128, 128))
    b2 = rng.normal(0, 0.1, 128)
    W3 = rng.normal(0, 0.1, (288, 128))
    b3 = rng.normal(0, 0.1, 288)
    W3[mo.PAD] = 0
    b3[mo.PAD] = 0
    return [W1, W2, b2, W3, b3]


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    x = np.concatenate([rng.normal(size=(16, 7)), np.ones((16, 1))], 1)
    t = rng.normal(size=(16, 288))
    t[:, mo.PAD] = 0
    loss, g = mo.loss_and_grads(x, t, p, emulate_bf16=False)
    eps = 1e-6
    for which, idx in ((0, (3, 7)), (0, (100, 2)), (1, (5, 77)), (2, (9,)), (3, (17, 40)), (3, (200, 3)),
                       (4, (150,))):
        q = [a.copy() for a in p]
        q[which][idx] += eps
        lp, _ = mo.loss_and_grads(x, t, q, emulate_bf16=False)
        q[which][idx] -= 2 * eps
        lm, _ = mo.loss_and_grads(x, t, q, emulate_bf16=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[which][idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (which, idx, fd, g[which][idx])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 65504.0, 1e-30], dtype=np.float32)
    r = mo.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even
    assert r[2] == 1.0 + 2 ** -7                  # above the tie rounds up
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8)
