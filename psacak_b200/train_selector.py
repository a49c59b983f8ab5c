"""Trains the schedule selector on timings the builder records itself.

    python -m psacak_b200.train_selector --texts 160 --out psacak_b200/models/selector.npz

Training texts follow the serving mix (lengths log-uniform on [4 KiB, 64 MiB]
symbols, half u8 ACGT, half u32 over 2^16, generated on the device), plus a
quarter as many genome-like u8 texts (order-3 Markov with N runs and long
mutated copies, 64 KiB .. 64 MiB) so that the model sees what long repeats
cost the prefix-doubling schedules; each is autotuned exhaustively (every
schedule timed with CUDA events), the statistics kernel gives its features,
and the MLP is fitted to log2(ms) on the GPU.  A held-out quarter measures regret against the exhaustive best,
beside the fixed default schedule; the report is printed as JSON and saved
next to the model.
"""
import argparse
import json
import os
import sys
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--texts", type=int, default=160)
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "models",
                                                  "selector.npz"))
    args = ap.parse_args(argv)
    import torch
    import psacak_b200 as pk
    from psacak_b200 import selector as sel
    from psacak_b200 import serve

    from psacak_b200 import synth
    ctx = pk.Context(0)
    plan = serve.request_plan(args.texts, args.seed)
    genome = [(int(m), 0, args.seed + 1000 + i)
              for i, m in enumerate(synth.loguniform(args.texts // 4, 64 << 10, 64 << 20, args.seed + 1))]
    maxn = max(n for n, _, _ in plan + genome)
    d_text = torch.empty(maxn * 4, dtype=torch.uint8, device="cuda")
    d_sa = torch.empty(maxn, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    X, T = [], []
    t0 = time.perf_counter()
    for i, (n, w, s) in enumerate(plan + genome):
        if w == 0:  # genome-like bytes, generated on the host
            w = 1
            d_text[:n].copy_(torch.from_numpy(synth.genome(n, seed=s)))
        else:
            serve.make_text(ctx, d_text.data_ptr(), n, w, s, stream.cuda_stream)
        torch.cuda.synchronize()
        X.append(sel.features(ctx, d_text.data_ptr(), n, w))
        T.append(sel.autotune(ctx, d_text.data_ptr(), n, w, d_sa.data_ptr(), reps=2))
    X, T = np.array(X, np.float32), np.array(T)
    t_tune = time.perf_counter() - t0
    rng = np.random.default_rng(args.seed)
    perm = rng.permutation(len(X))
    nte = max(1, len(X) // 4)
    te, tr = perm[:nte], perm[nte:]
    Tl, M = sel.targets(T)
    net = sel.Selector(ctx, seed=args.seed)
    hist = net.train(X[tr], Tl[tr], M[tr], epochs=args.epochs, lr=args.lr)
    picks = np.array([net.predict(x)[0] for x in X[te]])
    best = T[te].min(axis=1)
    reg_sel = T[te, picks] / best - 1
    reg_def = T[te, sel.DEFAULT_INDEX] / best - 1
    report = {
        "texts": len(X), "train": len(tr), "held_out": len(te), "autotune_seconds": t_tune,
        "loss_first": hist[0], "loss_last": hist[-1],
        "held_out_ms": {"best": float(best.sum()), "selector": float(T[te, picks].sum()),
                        "default": float(T[te, sel.DEFAULT_INDEX].sum())},
        "regret_selector_mean": float(reg_sel.mean()), "regret_default_mean": float(reg_def.mean()),
        "schedules": sel.SCHEDULES,
    }
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    net.save(args.out, meta=report)
    np.savez(os.path.splitext(args.out)[0] + "_data.npz", X=X, T=T)
    with open(os.path.splitext(args.out)[0] + "_report.json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
