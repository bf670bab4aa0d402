"""The CPU restatement of the warm-start network, checked by finite differences (no GPU)."""
import numpy as np

from bigwhoop_b200 import ratemodel


def test_cpu_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = ratemodel.init_params(1).astype(np.float64)
    X = rng.random((12, 34))
    t = rng.random(12)
    g, _ = ratemodel.cpu_gradient(p, X, t)
    idx = rng.choice(p.size, 40, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = np.mean((ratemodel.cpu_forward(pp, X)[0] - t) ** 2)
        lm = np.mean((ratemodel.cpu_forward(pm, X)[0] - t) ** 2)
        assert abs((lp - lm) / (2 * h) - g[i]) < 1e-5 * max(1.0, abs(g[i])), i
