"""The schedule selector on the GPU: forward and backward kernels against the
CPU fp32 reference (tolerance rtol 1e-3 / atol 1e-5), training, inference,
statistics, and the gain of the trained network over the best fixed
schedule on held-out texts (every schedule gives the same SA)."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import selector as sel, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def test_forward_and_gradients_match_reference(ctx):
    rng = np.random.default_rng(1)
    k = len(sel.SCHEDULES)
    net = sel.Selector(ctx, k=k, seed=3)
    p = net.params.cpu().numpy()
    X = rng.standard_normal((53, sel.NF)).astype(np.float32)
    T = rng.standard_normal((53, k)).astype(np.float32)
    M = (rng.random((53, k)) > 0.25).astype(np.float32)
    _, Y, _, _ = net.forward(X)
    Yr, _, _, _ = sel.ref_forward(p, X, k)
    np.testing.assert_allclose(Y.cpu().numpy(), Yr, rtol=1e-3, atol=1e-5)
    loss, G = net.gradients(X, T, M)
    lr_, gr = sel.ref_gradients(p, X, T, M, k)
    assert abs(loss - lr_) <= 1e-3 * max(1.0, abs(lr_))
    np.testing.assert_allclose(G.cpu().numpy(), gr, rtol=1e-3, atol=1e-5)


def test_training_fits_and_inference_is_argmin(ctx):
    rng = np.random.default_rng(2)
    k = 6
    X = rng.standard_normal((200, sel.NF)).astype(np.float32)
    X[:, -1] = 1.0
    W = rng.standard_normal((sel.NF, k)).astype(np.float32) * 0.5
    T = (np.tanh(X @ W) * 2.0).astype(np.float32)
    net = sel.Selector(ctx, k=k, seed=4)
    hist = net.train(X, T, np.ones_like(T), epochs=600, lr=3e-3)
    assert hist[-1] < 0.25 * hist[0]
    _, Y, _, _ = net.forward(X[:20])
    Y = Y.cpu().numpy()
    for i in range(20):
        c, pred = net.predict(X[i])
        np.testing.assert_allclose(pred, Y[i], rtol=1e-4, atol=1e-5)
        assert c == int(np.argmin(pred))


def test_text_statistics(ctx):
    t = synth.iid(1 << 20, b"ACGT", seed=7)
    d = torch.from_numpy(t).cuda()
    f = sel.features(ctx, d.data_ptr(), t.size, 1)
    assert f.shape == (16,) and f[-1] == 1.0
    assert abs(f[0] - np.log2(t.size + 1) / 32) < 1e-5 and f[1] == 0.25
    assert 0.2 < f[3] < 0.45          # LMS density of i.i.d. ACGT (~1/3)
    assert 0.15 < f[5] < 0.35         # equal neighbours (~1/4)
    rep = np.tile(synth.iid(4096, b"ACGT", seed=8), 64)
    fr = sel.features(ctx, torch.from_numpy(rep).cuda().data_ptr(), rep.size, 1)
    assert fr[6] > f[6]               # repeats are seen


def test_selector_beats_the_best_fixed_schedule(ctx):
    """What the trained network gains over the method without it.  Byte
    texts with long repeats (genome-like: mutated copies of earlier stretches)
    sort fastest by induced sorting at the top level (a recursion cut-off
    below their length): prefix doubling from the text needs a round per
    doubling of the longest repeat.  Integer texts with short repeats (i.i.d.
    over 2^16) sort fastest by prefix doubling from the text (a cut-off above
    their length), done in a few rounds.  With both kinds at the same lengths
    (16..40 Mi symbols) no single schedule suits both, so the best fixed one
    (the smallest total time on the training texts) loses on one kind; the
    network, reading the symbol width and the repeat statistics, picks per
    text.  Held-out texts: the selector's total time must be below the best
    fixed schedule's by at least 10%, and picks build the oracle's SA."""
    rng = np.random.default_rng(5)

    def text(kind, n, seed):
        if kind == 1:
            return synth.genome(n, seed=seed)
        return np.random.default_rng(seed).integers(0, 1 << 16, n, dtype=np.uint32)

    def texts(count, seed):
        return [(text(1 if i % 2 == 0 else 4, int(np.exp(rng.uniform(np.log(16 << 20), np.log(40 << 20)))),
                      seed + i), 1 if i % 2 == 0 else 4) for i in range(count)]

    def measure(items):
        X, Tm = [], []
        for t, w in items:
            d = torch.from_numpy(t.view(np.uint8)).cuda()
            sa = torch.empty(t.size, dtype=torch.int32, device="cuda")
            X.append(sel.features(ctx, d.data_ptr(), t.size, w))
            Tm.append(sel.autotune(ctx, d.data_ptr(), t.size, w, sa.data_ptr(), reps=2))
        return np.array(X), np.array(Tm)

    Xtr, Ttr = measure(texts(24, 100))
    Xte, Tte = measure(texts(12, 900))
    best_fixed = int(np.argmin(Ttr.sum(axis=0)))
    T, M = sel.targets(Ttr)
    net = sel.Selector(ctx, k=len(sel.SCHEDULES), seed=6)
    net.train(Xtr, T, M, epochs=1500, lr=3e-3)
    picks = [net.predict(x)[0] for x in Xte]
    sel_ms = sum(Tte[i, p] for i, p in enumerate(picks))
    fixed_ms = Tte[:, best_fixed].sum()
    best_ms = Tte.min(axis=1).sum()
    print("held-out: per-text best %.2f ms, selector %.2f ms, best fixed (%s) %.2f ms"
          % (best_ms, sel_ms, sel.SCHEDULES[best_fixed], fixed_ms))
    for i in range(len(Tte)):
        print("  text %d: best %.2f (#%d), pick %.2f (#%d), fixed %.2f" % (
            i, Tte[i].min(), int(Tte[i].argmin()), Tte[i, picks[i]], picks[i], Tte[i, best_fixed]))
    assert sel_ms <= 0.9 * fixed_ms
    # the picks for short texts of both kinds build the oracle's suffix arrays
    for w, n in ((1, 1 << 20), (4, 1 << 18)):
        t = text(w, n, 7000 + w)
        d = torch.from_numpy(t.view(np.uint8)).cuda()
        sa = torch.empty(t.size, dtype=torch.int32, device="cuda")
        p, _ = net.predict(sel.features(ctx, d.data_ptr(), t.size, w))
        sel.build(ctx, d.data_ptr(), t.size, w, sa.data_ptr(), 0, sel.SCHEDULES[p])
        torch.cuda.synchronize()
        want = o.psacak8(t) if w == 1 else o.psacak32(t)
        assert (sa.cpu().numpy().view(np.uint32) == want).all()
