"""The double-precision oracle of the learned-index trainer's gradient
(dL/dq for q = knot logits, output weights, output bias) against central
finite differences of its own loss.  The device trainer's gradient is
compared with this oracle in tests/test_gpu_parity.py."""
import numpy as np
import pytest

from oracle import oracle as o


def _random_q(rng):
    return np.concatenate([rng.normal(0, 0.8, 16), np.abs(rng.normal(1 / 16, 0.05, 16)), [rng.normal(0, 0.1)]])


@pytest.mark.parametrize("seed", range(6))
def test_grad_q_oracle_matches_central_differences(seed):
    rng = np.random.default_rng(seed)
    q = _random_q(rng) if seed else np.concatenate([np.zeros(16), np.full(16, 1 / 16), [0.0]])  # seed 0: identity
    n = int(rng.integers(50, 300))
    x = rng.random(n).astype(np.float32)
    t = np.sort(rng.random(n)).astype(np.float32)
    loss, g = o.learned_grad_q(q, x, t)
    assert abs(loss - o.learned_loss_q(q, x, t)) <= 1e-15
    eps = 1e-7  # samples within ~eps of a ramp end would bend the difference; with n <= 300 that is rare
    fd = np.empty_like(g)
    for i in range(len(q)):
        qp, qm = q.copy(), q.copy()
        qp[i] += eps
        qm[i] -= eps
        fd[i] = (o.learned_loss_q(qp, x, t) - o.learned_loss_q(qm, x, t)) / (2 * eps)
    scale = max(1e-12, float(np.abs(g).max()))
    assert np.abs(fd - g).max() <= 1e-6 * scale


def test_grad_q_softmax_direction():
    """Shifting every knot logit by the same amount leaves the widths, and the
    loss, unchanged: the logit gradient sums to zero."""
    rng = np.random.default_rng(9)
    q = _random_q(rng)
    x = rng.random(500).astype(np.float32)
    t = np.sort(rng.random(500)).astype(np.float32)
    _, g = o.learned_grad_q(q, x, t)
    assert abs(g[:16].sum()) <= 1e-9 * max(1e-12, np.abs(g[:16]).max())
