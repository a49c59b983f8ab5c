"""Trains the schedule selector on timings the builder records itself.

    python -m psacak_b200.train_selector --texts 240 --out psacak_b200/models/selector.npz

Training texts are requests of the serving mix (psacak_b200.serve: lengths
log-uniform on [4 KiB, 64 MiB] symbols; u8 ACGT i.i.d. and genome-like, u32
over 2^16 i.i.d. and Zipf with planted repeats).  Each is autotuned
exhaustively -- every schedule of selector.SCHEDULES timed with CUDA events,
and the library's default schedule beside them -- the statistics kernel
gives its features, and the MLP is fitted to log2(ms) on the GPU by the
library's forward / backward / Adam kernels.

A held-out quarter of the texts measures what the network gains.  Its picks
are compared with the per-text best (exhaustive autotune), with the best
fixed schedule -- the one schedule with the smallest total time on the
training texts -- and with the library's default schedule.  The report is
printed as JSON and saved next to the model.
"""
import argparse
import json
import os
import sys
import time

import numpy as np


def collect(ctx, plan, pool, log=None):
    """Features, per-schedule times and library-default times of the
    planned texts."""
    import torch
    from psacak_b200 import selector as sel
    from psacak_b200 import serve
    maxn = max(n for n, _, _ in plan)
    d_text = torch.empty(maxn * 4, dtype=torch.uint8, device="cuda")
    d_sa = torch.empty(maxn, dtype=torch.int32, device="cuda")
    X, T, D = [], [], []
    for i, (n, c, s) in enumerate(plan):
        w = serve.width_of(c)
        t = pool.text(n, c, s)
        d_text[:n * w].copy_(torch.from_numpy(t.view(np.uint8)))
        torch.cuda.synchronize()
        X.append(sel.features(ctx, d_text.data_ptr(), n, w))
        T.append(sel.autotune(ctx, d_text.data_ptr(), n, w, d_sa.data_ptr(), reps=2))
        D.append(sel.autotune(ctx, d_text.data_ptr(), n, w, d_sa.data_ptr(), reps=2, schedules=[None])[0])
        if log and (i + 1) % 40 == 0:
            log("autotuned %d/%d" % (i + 1, len(plan)))
    return np.array(X, np.float32), np.array(T), np.array(D)


def evaluate(T, D, picks, best_fixed):
    """Held-out totals and regrets of the selector's picks, the best fixed
    schedule and the library default."""
    best = T.min(axis=1)
    rows = np.arange(len(T))
    out = {"held_out_ms": {"per_text_best": float(best.sum()), "selector": float(T[rows, picks].sum()),
                           "best_fixed": float(T[:, best_fixed].sum()), "library_default": float(D.sum())}}
    for name, t in (("selector", T[rows, picks]), ("best_fixed", T[:, best_fixed]), ("library_default", D)):
        r = t / best - 1.0
        out["regret_" + name] = {"mean": float(r.mean()), "p50": float(np.percentile(r, 50)),
                                 "p90": float(np.percentile(r, 90)), "max": float(r.max())}
    out["selector_over_best_fixed_time"] = out["held_out_ms"]["selector"] / out["held_out_ms"]["best_fixed"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--texts", type=int, default=240)
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--data", default="", help="reuse features and timings from this .npz instead of timing")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "models",
                                                  "selector.npz"))
    args = ap.parse_args(argv)
    import psacak_b200 as pk
    from psacak_b200 import selector as sel
    from psacak_b200 import serve

    ctx = pk.Context(0)
    t0 = time.perf_counter()
    if args.data:
        d = np.load(args.data)
        X, T, D = d["X"], d["T"], d["D"]
    else:
        plan = serve.request_plan(args.texts, args.seed)
        pool = serve.TextPool(max(n for n, _, _ in plan), args.seed)
        X, T, D = collect(ctx, plan, pool, log=lambda m: print(m, flush=True))
    t_tune = time.perf_counter() - t0
    rng = np.random.default_rng(args.seed)
    perm = rng.permutation(len(X))
    nte = max(1, len(X) // 4)
    te, tr = perm[:nte], perm[nte:]
    best_fixed = int(np.argmin(T[tr].sum(axis=0)))
    Tl, M = sel.targets(T)
    net = sel.Selector(ctx, k=T.shape[1], seed=args.seed)
    hist = net.train(X[tr], Tl[tr], M[tr], epochs=args.epochs, lr=args.lr)
    picks = np.array([net.predict(x)[0] for x in X[te]])
    report = {"texts": len(X), "train": len(tr), "held_out": len(te), "autotune_seconds": t_tune,
              "loss_first": hist[0], "loss_last": hist[-1], "best_fixed_index": best_fixed,
              "best_fixed_schedule": sel.SCHEDULES[best_fixed], "library_default": {"u8": sel.library_default(1), "u32": sel.library_default(4)},
              "schedules": sel.SCHEDULES}
    report.update(evaluate(T[te], D[te], picks, best_fixed))
    # the same comparison over all texts (the network saw three quarters of them)
    all_picks = np.array([net.predict(x)[0] for x in X])
    report["all_texts"] = evaluate(T, D, all_picks, best_fixed)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out, meta=report)
    np.savez(os.path.splitext(args.out)[0] + "_data.npz", X=X, T=T, D=D)
    with open(os.path.splitext(args.out)[0] + "_report.json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
