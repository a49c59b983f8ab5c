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


def test_library_default_matches_the_header():
    """selector.library_default (the schedule a NULL psacak_schedule stands
    for, used as the yardstick of the selector's regret) equals the header's
    default cut-offs and tile size for both symbol widths."""
    import os
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "psacak_b200.h")
    text = open(hdr).read()

    def define(name):
        m = re.search(r"#define %s \((\d+)u << (\d+)\)" % name, text) or \
            re.search(r"#define %s (\d+)u\b" % name, text)
        assert m, name
        return int(m.group(1)) << int(m.group(2)) if m.lastindex == 2 else int(m.group(1))

    for width, name in ((1, "PSACAK_DEFAULT_FINISH_BELOW"), (4, "PSACAK_DEFAULT_FINISH_BELOW32")):
        d = sel.library_default(width)
        assert d["finish_below"] == define(name), (width, d)
        assert d["inner_finish_below"] == define("PSACAK_DEFAULT_INNER_FINISH_BELOW")
        assert d["tile_items"] == define("PSACAK_DEFAULT_TILE_ITEMS")
