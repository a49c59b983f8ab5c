"""The CPU fp32 reference of the selector network, pinned by finite
differences (it is the oracle the GPU gradients are checked against)."""
import numpy as np

from psacak_b200 import selector as sel


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    k = 5
    n = sel.NF * sel.NH + sel.NH + sel.NH * sel.NH + sel.NH + sel.NH * k + k
    p = (rng.standard_normal(n) * 0.2).astype(np.float64)
    X = rng.standard_normal((7, sel.NF))
    T = rng.standard_normal((7, k))
    M = (rng.random((7, k)) > 0.3).astype(np.float64)

    def loss_of(q):
        Y, _, _, _ = sel.ref_forward(q.astype(np.float32), X, k)
        return float(np.sum(M * (Y - T) ** 2) / M.sum())

    _, g = sel.ref_gradients(p.astype(np.float32), X, T.astype(np.float32), M.astype(np.float32), k)
    idx = rng.choice(n, 40, replace=False)
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-3
        fd = (loss_of(p + e) - loss_of(p - e)) / 2e-3
        assert abs(fd - g[i]) <= 2e-2 * max(1.0, abs(fd)), (i, fd, g[i])
