"""Serving loop: suffix-array build requests arriving as a Poisson process,
served from host buffers by worker threads, with learned schedule selection.

Requests: lengths log-uniform on [lo, hi] symbols (4 KiB .. 64 MiB by
default), a quarter each of
* u8 ACGT, i.i.d. uniform;
* u8 ACGT, genome-like (order-3 Markov, N runs, long mutated copies);
* u32 over 2^16, i.i.d. uniform;
* u32 over 2^16, Zipf(1.1) with 10% planted repeats of 1K..100K symbols.
A request's text is a window of one of a few long texts per class generated
on the host up front (a window of such a text follows the same law), handed
to the server as a pageable host array; its suffix array goes back to a
host buffer.

Serving: an arrival thread releases the requests at Poisson times; each of
`workers` threads owns a builder context, a CUDA stream and device and
pinned host buffers, takes the oldest waiting request and serves it:
upload the text -> statistics kernel -> selector inference kernel ->
suffix-array build with the chosen schedule -> download the suffix array.
Two workers overlap one request's transfers with another's build.  Latency
is measured per request by wall clock from its arrival time to the moment
its suffix array is in host memory.

The arrival rate is `load` x the capacity measured first with the same
workers kept busy (closed loop over the first requests of the plan, after
one untimed pass over the same requests).
Regret against exhaustive autotuning over every schedule is measured
afterwards on a sample of the requests, for the selector's picks, the best
fixed schedule of the training data, and the library's default schedule.
"""
import math
import queue
import threading
import time

import numpy as np

from . import synth
from . import selector as sel

CLASSES = ("acgt_iid", "acgt_genome", "u32_iid", "u32_zipf")


def width_of(cls):
    return 1 if cls.startswith("acgt") else 4


def class_text(cls, n, seed):
    """A host text of class `cls` with n symbols."""
    if cls == "acgt_iid":
        return synth.iid(n, b"ACGT", seed=seed)
    if cls == "acgt_genome":
        return synth.genome(n, seed=seed)
    if cls == "u32_iid":
        return np.random.default_rng(seed).integers(0, 1 << 16, n, dtype=np.uint32)
    if cls == "u32_zipf":
        return synth.zipf32(n, alphabet=1 << 16, s=1.1, repeat_frac=0.10, rep_min=1000, rep_max=100000, seed=seed)
    raise ValueError(cls)


def request_plan(count, seed, lo=4 << 10, hi=64 << 20):
    """[(n, class, text seed)] for `count` requests."""
    lens = synth.loguniform(count, lo, hi, seed)
    return [(int(n), CLASSES[synth.hash2(seed, i) & 3], synth.hash2(seed + 1, i)) for i, n in enumerate(lens)]


class TextPool:
    """`copies` long host texts per class; request i reads a window of one
    of them (chosen and placed by its seed)."""

    def __init__(self, max_len, seed, copies=2):
        self.max_len = max_len
        self.texts = {c: [class_text(c, max_len, synth.hash2(seed + 17 * k, j)) for j in range(copies)]
                      for k, c in enumerate(CLASSES)}

    def text(self, n, cls, s):
        pool = self.texts[cls]
        t = pool[s % len(pool)]
        off = (s >> 8) % (self.max_len - n + 1)
        return t[off:off + n]


class Worker:
    """One serving thread's resources: context, stream, buffers."""

    def __init__(self, device, max_n, net):
        import torch
        import psacak_b200 as pk
        self.torch = torch
        self.ctx = pk.Context(device)
        self.stream = torch.cuda.Stream(device=device)
        self.d_text = torch.empty(max_n * 4, dtype=torch.uint8, device="cuda")
        self.d_sa = torch.empty(max_n, dtype=torch.int32, device="cuda")
        self.h_sa = torch.empty(max_n, dtype=torch.int32, pin_memory=True)
        self.net = net.bind(self.ctx) if net is not None else None

    def pick(self, n, w):
        f = sel.features(self.ctx, self.d_text.data_ptr(), n, w)
        if self.net is None:
            return None, None
        c = self.net.predict(f)[0]
        return c, sel.SCHEDULES[c]

    def serve(self, text, w, schedule="select"):
        """Builds the suffix array of a host text; returns (host SA view,
        schedule index or None)."""
        torch = self.torch
        n = text.size
        src = torch.from_numpy(text.view(np.uint8))
        with torch.cuda.stream(self.stream):
            self.d_text[:src.numel()].copy_(src)
        self.stream.synchronize()
        if schedule == "select":
            c, sc = self.pick(n, w)
        else:
            c, sc = None, schedule
        sel.build(self.ctx, self.d_text.data_ptr(), n, w, self.d_sa.data_ptr(), self.stream.cuda_stream, sc)
        with torch.cuda.stream(self.stream):
            self.h_sa[:n].copy_(self.d_sa[:n], non_blocking=True)
        self.stream.synchronize()
        return self.h_sa.numpy()[:n].view(np.uint32), c

    def close(self):
        self.ctx.close()


def _closed_loop(workers, items):
    """Serves `items` [(text, w)] with every worker busy; returns seconds."""
    q = queue.Queue()
    for it in items:
        q.put(it)

    def loop(wk):
        while True:
            try:
                t, w = q.get_nowait()
            except queue.Empty:
                return
            wk.serve(t, w)

    ths = [threading.Thread(target=loop, args=(wk,)) for wk in workers]
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return time.perf_counter() - t0


def run(net, count=20000, seed=5, load=0.7, workers=2, autotune_sample=200, lo=4 << 10, hi=64 << 20,
        best_fixed=None, probe=300, device=0, log=None, check=None):
    """Runs the serving loop; returns the report dict.  `check(i, text, sa)`
    (optional) is called after the timed run on a few requests of at most
    1 MiB symbols, served again the same way, to compare with an oracle."""
    import torch
    plan = request_plan(count, seed, lo, hi)
    t_pool = time.perf_counter()
    pool = TextPool(hi, seed)
    pool_s = time.perf_counter() - t_pool
    maxn = max(n for n, _, _ in plan)
    ws = [Worker(device, maxn, net) for _ in range(workers)]
    # warm-up: every worker builds a few requests (workspace, module loading)
    for wk in ws:
        for n, c, s in plan[:4]:
            wk.serve(pool.text(n, c, s), width_of(c))
    # capacity with every worker busy: the probe requests twice, the first
    # pass loading every kernel the picks use and growing each worker's
    # workspace to the probe's largest request, the second one timed
    pr = plan[:min(probe, count)]
    items = [(pool.text(n, c, s), width_of(c)) for n, c, s in pr]
    _closed_loop(ws, items)
    secs = _closed_loop(ws, items)
    capacity = len(pr) / secs
    lam = load * capacity
    rng = np.random.default_rng(seed + 7)
    arrivals = np.cumsum(rng.exponential(1.0 / lam, count))
    start = np.zeros(count)
    finish = np.zeros(count)
    picks = np.full(count, -1, dtype=np.int64)
    who = np.zeros(count, dtype=np.int64)
    q = queue.Queue()
    t0 = time.perf_counter() + 0.05

    def arrive():
        for i in range(count):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            q.put(i)
        for _ in ws:
            q.put(None)

    def work(k, wk):
        while True:
            i = q.get()
            if i is None:
                return
            n, c, s = plan[i]
            start[i] = time.perf_counter() - t0
            text = pool.text(n, c, s)
            sa, pk_ = wk.serve(text, width_of(c))
            finish[i] = time.perf_counter() - t0
            picks[i] = -1 if pk_ is None else pk_
            who[i] = k
            if log and (i + 1) % 2000 == 0:
                log("served %d/%d" % (i + 1, count))

    ths = [threading.Thread(target=work, args=(k, wk)) for k, wk in enumerate(ws)]
    for th in ths:
        th.start()
    at = threading.Thread(target=arrive)
    at.start()
    at.join()
    for th in ths:
        th.join()
    latency = finish - arrivals
    wait = start - arrivals
    service = finish - start
    symbols = sum(n for n, _, _ in plan)
    makespan = finish.max() - arrivals[0]
    out = {
        "requests": count, "workers": workers, "load": load, "capacity_requests_per_s": capacity,
        "arrival_rate_per_s": lam, "text_pool_seconds": pool_s,
        "p50_latency_ms": 1000 * float(np.percentile(latency, 50)),
        "p99_latency_ms": 1000 * float(np.percentile(latency, 99)),
        "mean_latency_ms": 1000 * float(latency.mean()),
        "p50_wait_ms": 1000 * float(np.percentile(wait, 50)), "p99_wait_ms": 1000 * float(np.percentile(wait, 99)),
        "mean_service_ms": 1000 * float(service.mean()),
        "throughput_suffixes_per_s": symbols / makespan, "total_suffixes": symbols,
        "offered_suffixes_per_s": symbols / float(arrivals[-1] - arrivals[0]),
        "schedule_histogram": {str(k): int((picks == k).sum()) for k in range(len(sel.SCHEDULES))},
        "requests_per_worker": [int((who == k).sum()) for k in range(workers)],
    }
    if check is not None:
        small = [i for i in range(count) if plan[i][0] <= (1 << 20)][:8]
        res = []
        for i in small:
            n, c, s = plan[i]
            text = pool.text(n, c, s)
            sa, _ = ws[0].serve(text, width_of(c))
            res.append(bool(check(i, text, sa.copy())))
        out["checked_against_oracle"] = {"requests": len(res), "equal": int(sum(res))}
    # regret on a sample, against exhaustive autotuning over every schedule
    if autotune_sample:
        wk = ws[0]
        idx = np.random.default_rng(seed + 11).choice(count, min(autotune_sample, count), replace=False)
        reg = {"selector": [], "best_fixed": [], "library_default": []}
        for i in idx:
            n, c, s = plan[i]
            text = pool.text(n, c, s)
            w = width_of(c)
            src = torch.from_numpy(text.view(np.uint8))
            wk.d_text[:src.numel()].copy_(src)
            torch.cuda.synchronize()
            times = sel.autotune(wk.ctx, wk.d_text.data_ptr(), n, w, wk.d_sa.data_ptr(), reps=2)
            dflt = sel.autotune(wk.ctx, wk.d_text.data_ptr(), n, w, wk.d_sa.data_ptr(), reps=2,
                                schedules=[None])[0]
            best = times.min()
            if picks[i] >= 0:
                reg["selector"].append(times[picks[i]] / best - 1.0)
            if best_fixed is not None:
                reg["best_fixed"].append(times[best_fixed] / best - 1.0)
            reg["library_default"].append(dflt / best - 1.0)
        out["regret_sample"] = int(len(idx))
        for k, v in reg.items():
            if v:
                v = np.array(v)
                out["regret_" + k] = {"mean": float(v.mean()), "p50": float(np.percentile(v, 50)),
                                      "p90": float(np.percentile(v, 90)), "max": float(v.max())}
        if best_fixed is not None:
            out["best_fixed_schedule"] = sel.SCHEDULES[best_fixed]
    for wk in ws:
        wk.close()
    return out
