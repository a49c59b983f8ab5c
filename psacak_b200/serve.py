"""Serving loop with Poisson arrivals and learned schedule selection.

A stream of build requests -- lengths log-uniform on [lo, hi] symbols, half
u8 texts over ACGT and half u32 texts over 2^16 symbols -- is served FIFO by
one GPU.  Each request's text is generated on the device (its load is not
part of the service), then served as: statistics kernel -> selector
inference kernel -> suffix-array build with the chosen schedule.  Service
times are measured with CUDA events; arrivals are a Poisson process at
`load` x the measured capacity, and the FIFO queue is simulated from the
measured service times (start = max(arrival, previous finish)).

Reported: p50 / p99 latency, throughput (suffixes/s over the makespan), mean
service time, and regret against exhaustive autotuning on a sample of the
requests (regret = time of the chosen schedule / best time - 1), beside the
regret of the fixed default schedule.
"""
import math
import time

import numpy as np

from . import synth
from . import selector as sel

ACGT = b"ACGT"


def request_plan(count, seed, lo=4 << 10, hi=64 << 20):
    lens = synth.loguniform(count, lo, hi, seed)
    widths = [1 if (synth.hash2(seed, i) & 1) == 0 else 4 for i in range(count)]
    seeds = [synth.hash2(seed + 1, i) for i in range(count)]
    return [(int(n), w, s) for n, w, s in zip(lens, widths, seeds)]


def make_text(ctx, d_text, n, width, seed, stream):
    if width == 1:
        sel.gen_iid_dev(ctx, d_text, n, 1, ACGT, seed, stream)
    else:
        sel.gen_iid_dev(ctx, d_text, n, 4, 1 << 16, seed, stream)


def run(ctx, net, count=20000, seed=5, load=0.7, autotune_sample=200, lo=4 << 10, hi=64 << 20, log=None):
    import torch
    plan = request_plan(count, seed, lo, hi)
    maxn = max(n for n, _, _ in plan)
    d_text = torch.empty(maxn * 4, dtype=torch.uint8, device="cuda")
    d_sa = torch.empty(maxn, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    service = np.zeros(count)
    picks = np.zeros(count, dtype=np.int64)
    t_start = time.perf_counter()
    for i, (n, w, s) in enumerate(plan):
        make_text(ctx, d_text.data_ptr(), n, w, s, stream.cuda_stream)
        torch.cuda.synchronize()
        e0.record(stream)
        f = sel.features(ctx, d_text.data_ptr(), n, w)
        c = net.predict(f)[0] if net is not None else sel.DEFAULT_INDEX
        sel.build(ctx, d_text.data_ptr(), n, w, d_sa.data_ptr(), stream.cuda_stream, sel.SCHEDULES[c])
        e1.record(stream)
        torch.cuda.synchronize()
        service[i] = e0.elapsed_time(e1) / 1000.0
        picks[i] = c
        if log and (i + 1) % 2000 == 0:
            log("served %d/%d (%.1f s)" % (i + 1, count, time.perf_counter() - t_start))
    # Poisson arrivals at `load` x capacity, FIFO single server
    rng = np.random.default_rng(seed + 7)
    mean_s = float(service.mean())
    lam = load / mean_s
    arrivals = np.cumsum(rng.exponential(1.0 / lam, count))
    finish = np.zeros(count)
    prev = 0.0
    for i in range(count):
        start = max(arrivals[i], prev)
        prev = finish[i] = start + service[i]
    latency = finish - arrivals
    symbols = sum(n for n, _, _ in plan)
    makespan = finish[-1] - arrivals[0]
    out = {
        "requests": count, "load": load, "arrival_rate_per_s": lam, "mean_service_ms": 1000 * mean_s,
        "p50_latency_ms": 1000 * float(np.percentile(latency, 50)),
        "p99_latency_ms": 1000 * float(np.percentile(latency, 99)),
        "throughput_suffixes_per_s": symbols / makespan, "total_suffixes": symbols,
        "schedule_histogram": {str(k): int((picks == k).sum()) for k in range(len(sel.SCHEDULES))},
    }
    # regret on a sample, measured against exhaustive autotuning
    if autotune_sample:
        idx = np.random.default_rng(seed + 11).choice(count, min(autotune_sample, count), replace=False)
        reg_sel, reg_def = [], []
        for i in idx:
            n, w, s = plan[i]
            make_text(ctx, d_text.data_ptr(), n, w, s, stream.cuda_stream)
            torch.cuda.synchronize()
            times = sel.autotune(ctx, d_text.data_ptr(), n, w, d_sa.data_ptr(), reps=2)
            best = times.min()
            reg_sel.append(times[picks[i]] / best - 1.0)
            reg_def.append(times[sel.DEFAULT_INDEX] / best - 1.0)
        reg_sel, reg_def = np.array(reg_sel), np.array(reg_def)
        out["regret_sample"] = int(len(idx))
        out["regret_selector"] = {"mean": float(reg_sel.mean()), "p50": float(np.percentile(reg_sel, 50)),
                                  "p90": float(np.percentile(reg_sel, 90)), "max": float(reg_sel.max())}
        out["regret_default"] = {"mean": float(reg_def.mean()), "p50": float(np.percentile(reg_def, 50)),
                                 "p90": float(np.percentile(reg_def, 90)), "max": float(reg_def.max())}
    return out
