"""The CPU restatement of the warm-start network, checked by finite
differences (FP64, no BF16 rounding)."""
import numpy as np

from mlp_oracle import NIN, NPARAM, gradient


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.3, NPARAM)
    norm = np.concatenate([rng.normal(0, 1, NIN), rng.uniform(0.5, 2, NIN), [0.3, 1.7]])
    X = rng.normal(0, 1, (40, NIN))
    t = rng.normal(0, 1, 40)
    g, loss = gradient(w, norm, X, t, rnd=None)
    eps = 1e-6
    for i in rng.choice(NPARAM, 60, replace=False).tolist() + [NPARAM - 1]:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (gradient(wp, norm, X, t, rnd=None)[1] - gradient(wm, norm, X, t, rnd=None)[1]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
