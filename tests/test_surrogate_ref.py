"""The float64 CPU reference of the surrogate network: its hand-derived
backward pass against central finite differences (relative error < 1e-6 on
sampled weights of every layer)."""
import numpy as np

from tests import surrogate_ref as R


def test_reference_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    P = R.random_params(64, rng)
    x0, tgt = R.random_batch(1, rng)
    _, G = R.loss_and_grad(P, x0, tgt)
    h = 1e-6
    for name in ["w1", "w2", "w3", "w4", "w5", "b1", "b3", "b5"]:
        flat = P[name].reshape(-1)
        for idx in rng.choice(flat.size, 3, replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _ = R.loss_and_grad(P, x0, tgt)
            flat[idx] = old - h
            lm, _ = R.loss_and_grad(P, x0, tgt)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            an = G[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)) + 1e-12, (name, idx, fd, an)
