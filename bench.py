#!/usr/bin/env python
"""bench.py -- suffix-array construction throughput of psacak_b200 on B200.

Workload (default): psacak8 on a 1 GiB (2^30-byte) genome-like text -- an
order-3 Markov chain over ACGT with ~5% 'N' runs and ~30% of positions
copied from earlier segments with 1% point mutations (seed 2), u32 suffix
array.  One "step" is one complete build of that text.

Prints one JSON line (rank 0):
  value   suffixes/s with the text resident in HBM (device-timed, CUDA events
          on the build's stream, max over ranks);
  e2e     the same metric through the host-pointer C ABI (psacak8_ctx), the
          H2D copy of the text and the D2H copy of the SA inside each step;
  roofline  the dominant kernel's algorithmic bytes / its device time,
          measured live with the library's event profiler, against the
          measured HBM copy bandwidth;
  cpu_baseline  the CPU oracle (a C++ restatement of the reference's serial
          path) on a bounded window of the same text, one core;
  cpu_baseline_all_cores  the restatement of the reference's pipelined
          induced scans (fetch / induce / flush, src/pipeline.rs) on every
          host core, on a bounded prefix of the same text.

`--impl reference` times the pipelined restatement instead, on every host
core, one build of a bounded prefix of the workload text per step.
Multi-GPU (torchrun): every rank builds its own replica of the workload
(a single suffix array does not shard), "scaling": "weak".
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "suffixes/sec (psacak8 suffix-array build, bit-exact)"
UNIT = "suffixes/s"
GIB = 1 << 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--bytes", type=int, default=GIB, help="text length (default 2^30)")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=64 << 20,
                    help="bytes of the CPU samples (reference arm, 1-core and all-core baselines)")
    ap.add_argument("--engine", type=int, default=0, help="psacak_schedule.engine (0 = auto)")
    ap.add_argument("--profile-json", default="", help="also write per-kernel stats here")
    ap.add_argument("--workload", default="genome1g",
                    choices=["genome1g", "batch4096", "zipf32", "iid8m", "serve", "derived", "short20k"],
                    help="genome1g (default, the headline), batch4096 (4096 texts in one batched build), "
                         "zipf32 (psacak32 on 256M Zipf symbols), iid8m (8 MiB i.i.d. ACGT), "
                         "short20k (20,000 texts of 256 B..8 KiB in one batched build)")
    ap.add_argument("--requests", type=int, default=20000, help="serve: number of requests")
    ap.add_argument("--load", type=float, default=0.7, help="serve: arrival rate / measured capacity")
    ap.add_argument("--workers", type=int, default=2, help="serve: worker threads (one context each)")
    ap.add_argument("--regret-sample", type=int, default=200, help="serve: requests whose selector choice is checked against exhaustive autotune")
    ap.add_argument("--plain-texts", type=int, default=0,
                    help="batch4096: time the per-text loop on this many texts (0 = all)")
    ap.add_argument("--no-tune", action="store_true", help="batched forms: skip the autotuner (library default)")
    ap.add_argument("--no-batch", action="store_true",
                    help="genome1g: skip the batched form (4096 texts) that the default run reports beside it")
    ap.add_argument("--batch-steps", type=int, default=3,
                    help="genome1g: timed steps of the batched form (each ~0.7 s)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="genome1g: skip the exhaustive-autotune form of the headline text")
    ap.add_argument("--single-build", action="store_true",
                    help="build the workload once and exit (for ncu launch lists)")
    return ap.parse_args()


def workload_config(args):
    if args.workload == "short20k":
        return {"workload": "batched psacak8: 20000 independent texts, lengths log-uniform 256 B..8 KiB, "
                            "ACGT order-2 Markov (text i seeded by hash(seed, i)), one u32 SA per text "
                            "(each sorted by one CTA in shared memory)",
                "texts": 20000, "seed": args.seed, "engine": args.engine,
                "l2_policy": "~46 MB of texts + ~183 MB of SAs (larger than L2 together); no flush",
                "parallelism": "texts sharded across ranks (LPT)" if args.gpus > 1 else "single"}
    if args.workload == "batch4096":
        return {"workload": "batched psacak8: 4096 independent texts, lengths log-uniform 1 KiB..4 MiB, "
                            "ACGT order-2 Markov (text i seeded by hash(seed, i)), one u32 SA per text",
                "texts": 4096, "seed": args.seed, "engine": args.engine,
                "l2_policy": "inputs larger than L2 (~2 GiB of texts, ~8 GiB of SAs); no flush",
                "parallelism": "texts sharded across ranks (LPT)" if args.gpus > 1 else "single"}
    if args.workload == "zipf32":
        return {"workload": "psacak32 on 268435456 u32 symbols, alphabet 2^20, Zipf(1.1) frequencies, 10% planted "
                            "repeats of length 1K..100K, u32 SA", "n": 1 << 28, "seed": args.seed,
                "l2_policy": "inputs larger than L2 (1 GiB text + 1 GiB SA); no flush",
                "parallelism": "replicas" if args.gpus > 1 else "single"}
    if args.workload == "derived":
        return {"workload": "LCP array, BWT and inverse SA from the suffix array of the %d-byte genome-like text "
                            "(order-3 Markov ACGT, ~5%% N runs, ~30%% mutated copies); a step = the three arrays"
                            % args.bytes, "n": args.bytes, "seed": args.seed,
                "l2_policy": "inputs larger than L2 (1 GiB text + 4 GiB SA + 4 GiB out); no flush",
                "parallelism": "replicas" if args.gpus > 1 else "single"}
    if args.workload == "iid8m":
        return {"workload": "psacak8 on 8 MiB i.i.d. uniform ACGT, u32 SA", "n": 8 << 20, "seed": args.seed,
                "l2_policy": "8 MiB text + 32 MiB SA fit in L2; a 256 MiB buffer is written between steps",
                "parallelism": "replicas" if args.gpus > 1 else "single"}
    return {
        "workload": "psacak8, genome-like u8 text of %d bytes (order-3 Markov ACGT, ~5%% N runs, ~30%% mutated "
                    "copies), u32 SA" % args.bytes,
        "n": args.bytes,
        "seed": args.seed,
        "generator": "psacak_b200.synth.genome (xoshiro256**)",
        "l2_policy": "inputs larger than L2 (1 GiB text + 4 GiB SA per step vs 126 MB L2); no flush",
        "engine": args.engine,
        "parallelism": "replicas" if args.gpus > 1 else "single",
    }


def make_text(args):
    from psacak_b200 import synth
    return synth.genome(args.bytes, seed=args.seed)


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_build_bytes(trace, extra_translate=0):
    """Whole-build algorithmic bytes: sum over levels of (6w + 32) m + 28 n_lms."""
    b = 0
    for lv in trace:
        w = lv["width"]
        b += (6 * w + 32) * lv["m"] + 28 * lv["n_lms"]
    return b + extra_translate


# -- clocks ------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        med = float(np.median(sm)) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# -- CPU oracle ----------------------------------------------------------------
def cpu_baseline_all(text, window):
    """Pipelined restatement (all host cores) on the first `window` bytes."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    cores = os.cpu_count() or 1
    w = text[:window].copy()
    t0 = time.perf_counter()
    oracle_lib.psacak8_par(w, cores)
    dt = time.perf_counter() - t0
    return {"value": window / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "first %d bytes of the workload text, one build on %d threads: the reference's pipelined "
                      "induced scans (fetch / induce / flush over 128Ki blocks), its chunked parallel naming, "
                      "prefetching u32 scans on the inner levels; C++ restatement, the Rust crate is unbuildable "
                      "here" % (window, cores),
            "seconds": dt}


def cpu_baseline_single(text, window):
    """1-core oracle on the first `window` bytes of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    w = text[:window].copy()
    t0 = time.perf_counter()
    oracle_lib.psacak8(w)
    dt = time.perf_counter() - t0
    return {"value": window / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "first %d bytes of the workload text, one serial build (C++ restatement of the "
                      "reference's serial path; the Rust crate is unbuildable here)" % window,
            "seconds": dt}


def run_reference(args):
    """The reference's CPU path on the host cores: per step, one build of a
    bounded prefix of the workload text with the restatement of its pipelined
    induced scans on every core."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    from psacak_b200 import synth
    cores = os.cpu_count() or 1
    sample = min(args.cpu_sample, args.bytes)
    text = synth.genome(sample, seed=args.seed)  # the workload text's first `sample` bytes
    one = cpu_baseline_single(text, sample)  # the serial restatement on the same sample, one core
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle_lib.psacak8_par(text, cores)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    secs = sum(times)
    value = sample * len(times) / secs
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(len(times), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "per step, one build of the first %d bytes of the workload text on %d threads: "
                                   "the reference's pipelined induced scans (fetch / induce / flush, 128Ki blocks), "
                                   "its chunked parallel naming, prefetching u32 scans on the inner levels; C++ "
                                   "restatement of the reference (the Rust crate is unbuildable on this image)"
                                   % (sample, cores)},
        "cpu_baseline_one_core": one,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# -- GPU arm -------------------------------------------------------------------
def run_serve(args):
    """Config 5: Poisson stream of build requests served from host buffers by
    two worker threads, with the learned schedule selector."""
    import torch
    import psacak_b200 as pk
    from psacak_b200 import selector as sel
    from psacak_b200 import serve
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ctx = pk.Context(0)
    model = os.path.join(ROOT, "psacak_b200", "models", "selector.npz")
    net = sel.Selector.load(ctx, model) if os.path.exists(model) else None
    best_fixed = None
    rep = os.path.join(ROOT, "psacak_b200", "models", "selector_report.json")
    if os.path.exists(rep):
        with open(rep) as f:
            best_fixed = json.load(f).get("best_fixed_index")

    def check(i, text, sa):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        want = oracle_lib.psacak8(text) if text.dtype == np.uint8 else oracle_lib.psacak32(text)
        return bool(np.array_equal(sa, want))

    clocks = ClockSampler(0)
    clocks.start()
    res = serve.run(net, count=args.requests, seed=args.seed, load=args.load, workers=args.workers,
                    autotune_sample=args.regret_sample, best_fixed=best_fixed,
                    log=lambda m: print(m, file=sys.stderr, flush=True),
                    check=None if args.no_verify else check)
    clk = clocks.stop()
    line = {"metric": "serving throughput (suffixes/s) with p50/p99 latency, learned schedule selector",
            "value": res["throughput_suffixes_per_s"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/u32", "data": "synthetic",
            "config": {"workload": "%d requests, Poisson arrivals at %.0f%% of the capacity measured with the same "
                                   "%d workers busy, lengths log-uniform 4 KiB..64 MiB symbols, a quarter each of "
                                   "u8 ACGT i.i.d., u8 ACGT genome-like, u32 over 2^16 i.i.d., u32 over 2^16 Zipf "
                                   "with repeats; texts in pageable host memory, suffix arrays back to pinned host "
                                   "buffers, copies inside the latency" % (args.requests, 100 * args.load,
                                                                          args.workers),
                       "seed": args.seed,
                       "selector": "trained model" if net is not None else "none (library default schedule)"},
            "e2e": {"value": res["throughput_suffixes_per_s"], "unit": UNIT,
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "every request's text upload and SA download are inside its latency"},
            "clocks": clk, "serving": res}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_b200(args):
    if args.workload == "serve":
        return run_serve(args)
    if args.workload in ("batch4096", "short20k"):
        return run_batch(args)
    if args.workload == "zipf32":
        return run_zipf32(args)
    if args.workload == "derived":
        return run_derived(args)
    import torch
    import psacak_b200 as pk

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    if args.workload == "iid8m":
        from psacak_b200 import synth
        args.bytes = 8 << 20
        text = synth.iid(args.bytes, b"ACGT", seed=args.seed)
    else:
        text = make_text(args)
    n = text.size
    ctx = pk.Context(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if args.workload == "iid8m" else None
    # the plain form is the library's default schedule (a NULL schedule);
    # --engine picks a level-0 engine with every other field zero instead
    sched = None if args.engine == 0 else {"engine": args.engine}
    d_text = torch.from_numpy(text).to(dev)
    d_sa = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def build():
        ctx.psacak8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sched)

    if args.single_build:
        build()
        torch.cuda.synchronize(dev)
        print(json.dumps({"single_build": True, "n": n, "launches": ctx.kernel_launches()}), flush=True)
        ctx.close()
        return 0

    for _ in range(args.warmup):
        build()
    torch.cuda.synchronize(dev)
    verified = None
    if not args.no_verify:
        verified = ctx.check_sa8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream)
    trace = ctx.trace()

    # timed region
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    l0 = ctx.kernel_launches()
    rt0 = ctx.round_trips()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if flush is None:
        e0.record(stream)
        for _ in range(args.steps):
            build()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        step_ms_total = e0.elapsed_time(e1)
    else:
        # small input: flush L2 between steps, time only the builds
        step_ms_total = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            e0.record(stream)
            build()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            step_ms_total += e0.elapsed_time(e1)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    launches = (ctx.kernel_launches() - l0) // max(args.steps, 1)
    round_trips = (ctx.round_trips() - rt0) // max(args.steps, 1)
    clk = clocks.stop()
    ms = step_ms_total / args.steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1000.0)

    # roofline of the dominant kernel: one more build with the event profiler
    roofline, stats = _profile_roofline(ctx, build, torch, dev)
    build_bytes = algorithmic_build_bytes(trace)
    build_gbs = build_bytes / (ms / 1000.0) / 1e9

    def timed_steps(sc):
        """Device ms per build with schedule sc, timed as the plain form
        (warm-up builds first; L2 flushed between steps for small inputs)."""
        for _ in range(max(1, args.warmup)):
            ctx.psacak8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sc)
        torch.cuda.synchronize(dev)
        total = 0.0
        if flush is None:
            e0.record(stream)
            for _ in range(args.steps):
                ctx.psacak8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sc)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            total = e0.elapsed_time(e1)
        else:
            for _ in range(args.steps):
                flush.fill_(1)
                e0.record(stream)
                ctx.psacak8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sc)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                total += e0.elapsed_time(e1)
        return _max_over_ranks(torch, dist, dev, total / args.steps)

    # learned-schedule form: the selector picks a schedule from the text's
    # statistics (inference kernel), timed the same way as the plain form
    learned = None
    model = os.path.join(ROOT, "psacak_b200", "models", "selector.npz")
    net = None
    if os.path.exists(model) and not args.single_build:
        from psacak_b200 import selector as sel
        net = sel.Selector.load(ctx, model)
    if net is not None:
        feats = sel.features(ctx, d_text.data_ptr(), n, 1)
        choice, _ = net.predict(feats)
        lsched = dict(sel.SCHEDULES[choice])
        lms_ = timed_steps(lsched)
        lok = None if args.no_verify else ctx.check_sa8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream)
        learned = {"value": world * n / (lms_ / 1000.0), "unit": UNIT, "ms_per_step": lms_, "schedule": lsched,
                   "verified": lok, "hbm_gbs_algorithmic_build": build_bytes / (lms_ / 1000.0) / 1e9}
    # zero schedule: every field 0, SACA-K with recursion down to the last
    # level as the reference does (the default sorts short levels directly)
    zero = None
    if not args.single_build:
        zs = {"engine": 0}
        zr0 = ctx.round_trips()
        zms = timed_steps(zs)
        zrt = (ctx.round_trips() - zr0) // (max(1, args.warmup) + args.steps)
        zok = None if args.no_verify else ctx.check_sa8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream)
        zero = {"value": world * n / (zms / 1000.0), "unit": UNIT, "ms_per_step": zms, "schedule": zs,
                "host_round_trips_per_step": zrt, "verified": zok,
                "note": "every field 0: induced sorting and recursion on every level, as the reference"}
    # texts the default sorts by prefix doubling from the text: SACA-K's
    # induced sorting at the top level (either engine), prefix doubling from
    # the first reduced string on, timed as the plain form
    induced = None
    if not args.single_build and n < (1 << 24):
        induced = {}
        for name, eng in (("bucket_engine", 1), ("doubling_engine", 2)):
            isc = {"engine": eng, "tile_items": 16, "finish_below": 1, "inner_finish_below": 1 << 30}
            ir0 = ctx.round_trips()
            ims = timed_steps(isc)
            irt = (ctx.round_trips() - ir0) // (max(1, args.warmup) + args.steps)
            iok = None if args.no_verify else ctx.check_sa8_dev(d_text.data_ptr(), n, d_sa.data_ptr(),
                                                                stream.cuda_stream)
            induced[name] = {"value": world * n / (ims / 1000.0), "unit": UNIT, "ms_per_step": ims, "schedule": isc,
                             "host_round_trips_per_step": irt, "verified": iok}

    # autotuned form: exhaustive search over the selector's schedules on
    # this text (the selector's fallback and yardstick), timed as above
    autotuned = None
    if not args.no_autotune and not args.single_build:
        from psacak_b200 import autotune, selector as sel
        t0 = time.perf_counter()
        tf = autotune.device_timer(
            lambda sc: ctx.psacak8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sc))
        best_i, table = autotune.exhaustive(tf, sel.SCHEDULES)
        tune_s = time.perf_counter() - t0
        asched = dict(sel.SCHEDULES[best_i])
        ams = timed_steps(asched)
        aok = None if args.no_verify else ctx.check_sa8_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream)
        autotuned = {"value": world * n / (ams / 1000.0), "unit": UNIT, "ms_per_step": ams, "schedule": asched,
                     "verified": aok, "search": "exhaustive over %d schedules (min of 1 build each, after a "
                                                "warm-up build)" % len(sel.SCHEDULES),
                     "search_seconds": tune_s, "search_ms": table,
                     "hbm_gbs_algorithmic_build": build_bytes / (ams / 1000.0) / 1e9}
        if learned is not None:
            learned["regret_vs_autotuned"] = learned["ms_per_step"] / ams - 1.0
    if args.profile_json and rank == 0:
        with open(args.profile_json, "w") as f:
            json.dump({"stats": stats, "trace": trace, "ms_per_step": ms}, f, indent=1)

    # end to end through the host-pointer C ABI
    # end to end through the host-pointer C ABI: pageable buffers (a numpy
    # array stands for the Rust Vec of psacak_inplace, the reference-facing
    # call) as `e2e`, and pinned buffers beside it
    e2e = e2e_pinned = None
    if not args.no_e2e:
        import ctypes
        lib = pk.lib()
        want = None if args.no_verify else d_sa.cpu().numpy().view(np.uint32)

        def host_run(ht, hs, api):
            times = []
            for i in range(max(args.warmup, 1) + args.e2e_steps):  # the same warm-up as the device-resident steps
                if dist:
                    dist.barrier()
                t0 = time.perf_counter()
                rc = lib.psacak8_ctx(ctx.handle, ctypes.c_void_p(ht.ctypes.data), n,
                                     ctypes.c_void_p(hs.ctypes.data), pk._sched_ptr(sched))
                dt = time.perf_counter() - t0
                if rc != 0:
                    pk._raise(rc)
                if i >= max(args.warmup, 1):
                    times.append(dt)
            e2e_s = _max_over_ranks(torch, dist, dev, float(np.mean(times)))
            out = {"value": world * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n, "d2h_bytes_per_step": 4 * n,
                   "ms_per_step": 1000.0 * e2e_s, "api": api}
            if want is not None:
                # the host array (sent bucket part by bucket part during the
                # final scans) must equal the checked device-resident one
                out["verified"] = bool(verified) and bool(np.array_equal(hs, want))
            return out

        hp_text = np.ascontiguousarray(text)
        hp_sa = np.empty(n, dtype=np.uint32)
        e2e = host_run(hp_text, hp_sa, "psacak8_ctx (host pointers, pageable buffers: the psacak_inplace shape)")
        del hp_sa
        h_text = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        h_text.numpy()[:] = text
        h_sa = torch.empty(n, dtype=torch.int32, pin_memory=True)
        e2e_pinned = host_run(h_text.numpy(), h_sa.numpy().view(np.uint32),
                              "psacak8_ctx (host pointers, pinned buffers)")
        del h_text, h_sa

    # batched form (4096 texts of 1 KiB..4 MiB, about 2 GiB) on the same GPU:
    # autotuned chunk size / block shape, beside the per-text loop
    batched = None
    if args.workload == "genome1g" and not args.no_batch and not args.single_build:
        from psacak_b200 import batch as pb
        del d_text, d_sa
        torch.cuda.empty_cache()
        btexts = pb.batch_texts(count=4096, seed=args.seed)
        batched = measure_batch(args, torch, ctx, dev, dist, world, rank, btexts, args.batch_steps,
                                max(3, args.warmup), tune=not args.no_tune, e2e_steps=args.e2e_steps,
                                cpu=False)
        batched["config"] = {"workload": "batched psacak8: 4096 independent texts, lengths log-uniform "
                                         "1 KiB..4 MiB, ACGT order-2 Markov (text i seeded by hash(seed, i)), "
                                         "one u32 SA per text", "texts": 4096, "seed": args.seed,
                             "l2_policy": "inputs larger than L2 (~2 GiB of texts, ~8 GiB of SAs); no flush",
                             "parallelism": "texts sharded across ranks (LPT)" if world > 1 else "single"}
        batched["scaling"] = "strong"

    cpu = cpu_all = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # both on the same prefix, so that the two rates compare
        cpu = cpu_baseline_single(text, min(args.cpu_sample, n))
        cpu_all = cpu_baseline_all(text, min(args.cpu_sample, n))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": workload_config(args),
            "e2e": e2e, "e2e_pinned": e2e_pinned, "roofline": roofline, "learned_schedule": learned,
            "autotuned_schedule": autotuned,
            "batched": batched,
            "plain_schedule": {"schedule": sched if sched is not None else "NULL (library default)",
                               "note": "the value above"},
            "zero_schedule": zero, "induced_top_level": induced,
            "hbm_gbs_algorithmic_build": build_gbs,
            "build_algorithmic_bytes": build_bytes,
            "cpu_baseline": cpu, "cpu_baseline_all_cores": cpu_all, "clocks": clk, "gpu_launches": int(launches),
            "host_round_trips_per_step": int(round_trips),
            "verified": verified, "levels": [[lv["m"], lv["n_lms"], lv["k"]] for lv in trace],
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _dist_init(torch, world, local):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist


def _max_over_ranks(torch, dist, dev, x):
    if not dist:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _profile_roofline(ctx, build, torch, dev):
    ctx.profile_reset()
    ctx.profile(True)
    build()
    torch.cuda.synchronize(dev)
    ctx.profile(False)
    stats = ctx.profile_stats()
    total_ms = sum(s["ms"] for s in stats)
    peak, peak_kind = measured_peak_hbm()

    def gbs(s):
        return s["bytes"] / (s["ms"] / 1000.0) / 1e9 if s["bytes"] and s["ms"] else None

    # the dominant kernel is the class with the most device time among those
    # with an algorithmic byte model; the largest classes are listed beside it
    dom = max((s for s in stats if s["bytes"] > 0), key=lambda s: s["ms"])
    achieved = gbs(dom)
    classes = []
    for s in sorted(stats, key=lambda s: -s["ms"])[:8]:
        a = gbs(s)
        classes.append({"kernel": s["name"], "launches": s["launches"], "ms": s["ms"],
                        "share": s["ms"] / total_ms if total_ms else None,
                        "achieved_gbs": a, "frac": a / peak if a else None})
    return {"bound": "hbm", "kernel": dom["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": dominant_traffic(dom["name"], dom["items"] / max(dom["launches"], 1)),
            "launches": dom["launches"], "algorithmic_bytes_per_launch": dom["bytes"] / max(dom["launches"], 1),
            "avg_launch_ms": dom["ms"] / max(dom["launches"], 1),
            "share_of_profiled_time": dom["ms"] / total_ms if total_ms else None,
            "largest_classes": classes}, stats


def measure_batch(args, torch, ctx, dev, dist, world, rank, texts, steps, warmup, tune=True, plain_texts=0,
                  e2e_steps=3, base_sched=None, cpu=True):
    """Batched build of `texts` (this rank's share by LPT): device-resident
    suffixes/s over `steps` timed builds, the schedule chosen by the
    autotuner (coordinate descent over chunk size, tile shape, block shape,
    finish_below and engine, psacak_b200.autotune), the per-text loop
    ("plain"), the end-to-end form through psacak8_batch with pageable
    per-text host buffers, and the roofline of the dominant kernel."""
    import ctypes
    import psacak_b200 as pk
    from psacak_b200 import autotune
    from psacak_b200 import batch as pb

    lens = [t.size for t in texts]
    total_all = sum(lens)
    mine = pb.shard_lpt(lens, world)[rank]
    my_texts = [texts[i] for i in mine]
    buf, off = pb.pack(my_texts)
    n = int(buf.size)
    d_texts = torch.from_numpy(buf).to(dev)
    d_sas = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def build_with(sc):
        ctx.psacak8_batch_dev(d_texts.data_ptr(), off, d_sas.data_ptr(), stream.cuda_stream, sc)

    # the library's NULL schedule, spelled out (the autotuner's start point)
    default = {"engine": 1, "tile_items": 16, "scan_ctas_per_sm": 4, "batch_chunk_mib": 3072,
               "finish_below": 1 << 24, "inner_finish_below": 1 << 30}
    if base_sched:
        default.update(base_sched)
    tuned = None
    sched = dict(default)
    if tune:
        t0 = time.perf_counter()
        best, best_ms, table = autotune.coordinate_descent(autotune.device_timer(build_with), default)
        tuned = {"schedule": best, "ms": best_ms,
                 "default_ms": next(r["ms"] for r in table if r["schedule"] == default),
                 "evaluated": len(table), "seconds": time.perf_counter() - t0,
                 "search": "coordinate descent, one sweep over " + ", ".join(autotune.BATCH_ORDER)}
        sched = best

    def build():
        build_with(sched)

    for _ in range(warmup):
        build()
    torch.cuda.synchronize(dev)
    verified = None
    if not args.no_verify:
        verified = True
        for i in range(len(my_texts)):
            a, b = int(off[i]), int(off[i + 1])
            if b > a and not ctx.check_sa8_dev(d_texts.data_ptr() + a, b - a, d_sas.data_ptr() + 4 * a,
                                               stream.cuda_stream):
                verified = False
                break
    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    l0 = ctx.kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        build()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = (ctx.kernel_launches() - l0) // max(steps, 1)
    ms = _max_over_ranks(torch, dist, dev, e0.elapsed_time(e1) / steps)
    value = total_all / (ms / 1000.0)
    roofline, stats = _profile_roofline(ctx, build, torch, dev)

    # plain: the same texts, one psacak8_dev call each (library default schedule)
    k_plain = len(my_texts) if plain_texts <= 0 else min(plain_texts, len(my_texts))
    torch.cuda.synchronize(dev)
    p0 = time.perf_counter()
    for i in range(k_plain):
        a, b = int(off[i]), int(off[i + 1])
        if b > a:
            ctx.psacak8_dev(d_texts.data_ptr() + a, b - a, d_sas.data_ptr() + 4 * a, stream.cuda_stream, None)
    torch.cuda.synchronize(dev)
    plain_s = time.perf_counter() - p0
    plain_value = sum(int(off[i + 1] - off[i]) for i in range(k_plain)) / plain_s

    e2e = None
    if not args.no_e2e:
        h_sas = [np.empty(t.size, dtype=np.uint32) for t in my_texts]
        ptrs_t = (ctypes.c_void_p * len(my_texts))(*[t.ctypes.data for t in my_texts])
        ptrs_s = (ctypes.c_void_p * len(my_texts))(*[x.ctypes.data for x in h_sas])
        lens_c = (ctypes.c_uint64 * len(my_texts))(*[t.size for t in my_texts])
        times = []
        for i in range(max(warmup, 1) + e2e_steps):  # the same warm-up as the device-resident steps
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            rc = pk.lib().psacak8_batch(ctx.handle, ptrs_t, lens_c, len(my_texts), ptrs_s, pk._sched_ptr(sched))
            dt = time.perf_counter() - t0
            if rc != 0:
                pk._raise(rc)
            if i >= max(warmup, 1):
                times.append(dt)
        e2e_s = _max_over_ranks(torch, dist, dev, float(np.mean(times)))
        e2e = {"value": total_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n, "d2h_bytes_per_step": 4 * n,
               "ms_per_step": 1000.0 * e2e_s, "api": "psacak8_batch (host pointers, pageable per-text buffers)"}
        if not args.no_verify:
            # the host arrays must equal the checked device-resident ones
            dev_sa = d_sas.cpu().numpy().view(np.uint32)
            e2e["verified"] = bool(verified) and all(
                np.array_equal(h_sas[i], dev_sa[int(off[i]):int(off[i + 1])]) for i in range(len(my_texts)))
    cpu_line = None
    if cpu and rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        t0 = time.perf_counter()
        done = 0
        for t in my_texts:
            oracle_lib.psacak8(t)
            done += t.size
            if time.perf_counter() - t0 > 5.0:
                break
        dt = time.perf_counter() - t0
        cpu_line = {"value": done / dt, "unit": UNIT, "cores": 1, "kind": "port",
                    "sample": "oracle builds of the first %d bytes of the batch, text by text" % done}
    del d_texts, d_sas
    return {"value": value, "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "texts": len(texts), "total_bytes": total_all, "schedule": sched, "autotune": tuned,
            "e2e": e2e, "roofline": roofline,
            "plain": {"value": plain_value, "unit": UNIT, "texts": k_plain,
                      "api": "psacak8_dev per text, same device-resident texts, library default schedule"},
            "batched_over_plain": value / plain_value, "cpu_baseline": cpu_line, "clocks": clk,
            "gpu_launches": int(launches), "verified": verified}


def run_batch(args):
    """Config 4 (4096 texts of 1 KiB..4 MiB) or 20,000 short texts in one
    batched build, and the per-text loop beside it."""
    import torch
    import psacak_b200 as pk
    from psacak_b200 import batch as pb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = _dist_init(torch, world, local)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    base = {"engine": args.engine} if args.engine else {}
    if args.workload == "short20k":
        texts = pb.batch_texts(count=20000, lo=256, hi=8 << 10, seed=args.seed)
        # texts below the default prefix-doubling cutoff: each sorted by one CTA in shared memory
        base["finish_below"] = 1 << 16
    else:
        texts = pb.batch_texts(count=4096, seed=args.seed)
    ctx = pk.Context(local)
    r = measure_batch(args, torch, ctx, dev, dist, world, rank, texts, args.steps, args.warmup,
                      tune=not args.no_tune, plain_texts=args.plain_texts, e2e_steps=args.e2e_steps,
                      base_sched=base)
    if rank == 0:
        line = {"metric": METRIC + " -- batched", "value": r["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic", "config": workload_config(args)}
        line.update({k: v for k, v in r.items() if k not in ("value", "unit", "ms_per_step", "steps", "warmup")})
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_derived(args):
    """LCP array, BWT and inverse SA of the 1 GiB genome-like text from its
    suffix array (built once, untimed, checked on the device); each step
    makes the three arrays.  Parity: the same arrays for a 64 MiB prefix of
    the text against the CPU restatements (Kasai's LCP, the BWT definition)."""
    import torch
    import psacak_b200 as pk

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = _dist_init(torch, world, local)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.bytes
    text = make_text(args)
    ctx = pk.Context(local)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    dt = torch.from_numpy(text).to(dev)
    ds = torch.empty(n, dtype=torch.int32, device=dev)
    ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), s)
    sa_ok = ctx.check_sa8_dev(dt.data_ptr(), n, ds.data_ptr(), s)
    lcp = torch.empty(n, dtype=torch.int32, device=dev)
    isa = torch.empty(n, dtype=torch.int32, device=dev)
    bwt = torch.empty(n, dtype=torch.uint8, device=dev)
    fm = torch.empty(pk.fm_bytes(n), dtype=torch.uint8, device=dev)
    # FM-index queries: 2^20 patterns of 20 bytes, half taken from the text
    # (they occur), half random over ACGT
    qn, qm = 1 << 20, 20
    qrng = np.random.default_rng(args.seed + 3)
    qpos = qrng.integers(0, n - qm, qn // 2)
    pats = np.concatenate([text[(qpos[:, None] + np.arange(qm)[None, :])].reshape(-1),
                           np.frombuffer(b"ACGT", np.uint8)[qrng.integers(0, 4, (qn - qn // 2) * qm)]])
    dpat = torch.from_numpy(pats).to(dev)
    doff = torch.arange(0, (qn + 1) * qm, qm, dtype=torch.int64, device=dev)
    dranges = torch.empty(2 * qn, dtype=torch.int32, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    primary = [0]

    def step():
        ev[0].record(stream)
        ctx.lcp8_dev(dt.data_ptr(), n, ds.data_ptr(), lcp.data_ptr(), s)
        ev[1].record(stream)
        primary[0] = ctx.bwt8_dev(dt.data_ptr(), n, ds.data_ptr(), bwt.data_ptr(), s)
        ev[2].record(stream)
        ctx.isa_dev(ds.data_ptr(), n, isa.data_ptr(), s)
        ev[3].record(stream)
        ctx.fm_build_dev(bwt.data_ptr(), n, primary[0], fm.data_ptr(), s)
        ev[4].record(stream)
        ctx.fm_count_dev(fm.data_ptr(), bwt.data_ptr(), dpat.data_ptr(), doff.data_ptr(), qn, dranges.data_ptr(), s)
        ev[5].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    tl = tb = ti = tf = tq = 0.0
    for _ in range(args.steps):
        step()
        torch.cuda.synchronize(dev)
        tl += ev[0].elapsed_time(ev[1])
        tb += ev[1].elapsed_time(ev[2])
        ti += ev[2].elapsed_time(ev[3])
        tf += ev[3].elapsed_time(ev[4])
        tq += ev[4].elapsed_time(ev[5])
    clk = clocks.stop()
    ms = (tl + tb + ti) / args.steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # parity on a prefix the CPU restatements finish in seconds
    verified = None
    if rank == 0 and not args.no_verify:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        m = min(n, 64 << 20)
        tp = text[:m].copy()
        dtp = torch.from_numpy(tp).to(dev)
        dsp = torch.empty(m, dtype=torch.int32, device=dev)
        ctx.psacak8_dev(dtp.data_ptr(), m, dsp.data_ptr(), s)
        lp = torch.empty(m, dtype=torch.int32, device=dev)
        bp = torch.empty(m, dtype=torch.uint8, device=dev)
        ctx.lcp8_dev(dtp.data_ptr(), m, dsp.data_ptr(), lp.data_ptr(), s)
        prim = ctx.bwt8_dev(dtp.data_ptr(), m, dsp.data_ptr(), bp.data_ptr(), s)
        sap = dsp.cpu().numpy().view(np.uint32)
        want_b, want_p = oracle_lib.bwt(tp, sap)
        verified = bool(sa_ok and (lp.cpu().numpy().view(np.uint32) == oracle_lib.lcp(tp, sap)).all()
                        and prim == want_p and (bp.cpu().numpy() == want_b).all())
        # FM-index ranges of 64 of the full text's queries against binary
        # search on the full suffix array (host copy)
        sa_full = ds.cpu().numpy().view(np.uint32)
        rg = dranges.cpu().numpy().view(np.uint32).reshape(-1, 2)
        for q in list(range(0, qn, qn // 32)) + list(range(qn // 2, qn, qn // 32)):
            want = oracle_lib.sa_range8(text, sa_full, pats[q * qm:(q + 1) * qm])
            got = (int(rg[q, 0]), int(rg[q, 1]))
            if (want[1] > want[0] and got != want) or (want[1] == want[0] and got[1] != got[0]):
                verified = False
    if rank == 0:
        line = {
            "metric": "suffixes/sec (LCP array + BWT + inverse SA from a suffix array, bit-exact)",
            "value": world * n / (ms / 1000.0), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8/u32", "data": "synthetic", "config": workload_config(args),
            "per_array_ms": {"lcp": tl / args.steps, "bwt": tb / args.steps, "isa": ti / args.steps},
            "fm_index": {"build_ms": tf / args.steps, "build_gbs_algorithmic": 3.0 * n / (tf / args.steps) / 1e6,
                         "queries": qn, "pattern_bytes": qm, "count_ms": tq / args.steps,
                         "patterns_per_s": qn / (tq / args.steps / 1000.0),
                         "index_bytes": pk.fm_bytes(n),
                         "note": "build reads the BWT (n bytes) and writes the rank checkpoints (~2n bytes); a "
                                 "query is a backward search, one warp per pattern, 2 rank lookups per byte"},
            "clocks": clk, "verified": verified,
            "verification": "device SA check of the full text; LCP and BWT of its 64 MiB prefix equal to the CPU "
                            "restatements; 64 FM-index query ranges equal to binary search on the suffix array",
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_zipf32(args):
    """Config 3: psacak32 on 256M Zipf(1.1) symbols over 2^20 with planted repeats."""
    import ctypes
    import torch
    import psacak_b200 as pk
    from psacak_b200 import synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = _dist_init(torch, world, local)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = 1 << 28
    text = synth.zipf32(n, alphabet=1 << 20, s=1.1, repeat_frac=0.10, rep_min=1000, rep_max=100000, seed=args.seed)
    ctx = pk.Context(local)
    d_text = torch.from_numpy(text.view(np.int32)).to(dev)
    d_sa = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def build():
        ctx.psacak32_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        build()
    torch.cuda.synchronize(dev)
    verified = None if args.no_verify else ctx.check_sa32_dev(d_text.data_ptr(), n, d_sa.data_ptr(),
                                                              stream.cuda_stream)
    trace = ctx.trace()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    l0 = ctx.kernel_launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        build()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = (ctx.kernel_launches() - l0) // max(args.steps, 1)
    ms = _max_over_ranks(torch, dist, dev, e0.elapsed_time(e1) / args.steps)
    value = world * n / (ms / 1000.0)
    roofline, _ = _profile_roofline(ctx, build, torch, dev)

    def timed_form(sched, note):
        """The same build with another schedule, timed as the default form."""
        for _ in range(max(1, args.warmup)):
            ctx.psacak32_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sched)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.psacak32_dev(d_text.data_ptr(), n, d_sa.data_ptr(), stream.cuda_stream, sched)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        fms = _max_over_ranks(torch, dist, dev, e0.elapsed_time(e1) / args.steps)
        ok = None if args.no_verify else ctx.check_sa32_dev(d_text.data_ptr(), n, d_sa.data_ptr(),
                                                            stream.cuda_stream)
        return {"value": world * n / (fms / 1000.0), "unit": UNIT, "ms_per_step": fms, "schedule": sched,
                "verified": ok, "levels": [[lv["m"], lv["n_lms"], lv["k"]] for lv in ctx.trace()], "note": note}

    induced = timed_form({"tile_items": 16, "finish_below": 1 << 26, "inner_finish_below": 1 << 30},
                         "induced sorting (chain doubling) at the top level, prefix doubling from the first "
                         "reduced string on")
    zero = timed_form({}, "every field 0: induced sorting and recursion on every level, as the reference")
    e2e = None
    if not args.no_e2e:
        h_text = torch.empty(n, dtype=torch.int32, pin_memory=True)
        h_text.numpy()[:] = text.view(np.int32)
        h_sa = torch.empty(n, dtype=torch.int32, pin_memory=True)
        times = []
        for i in range(max(args.warmup, 1) + args.e2e_steps):  # the same warm-up as the device-resident steps
            t0 = time.perf_counter()
            rc = pk.lib().psacak32_ctx(ctx.handle, ctypes.c_void_p(h_text.data_ptr()), n,
                                       ctypes.c_void_p(h_sa.data_ptr()), None)
            dt = time.perf_counter() - t0
            if rc != 0:
                pk._raise(rc)
            if i >= max(args.warmup, 1):
                times.append(dt)
        e2e_s = _max_over_ranks(torch, dist, dev, float(np.mean(times)))
        e2e = {"value": world * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * n,
               "ms_per_step": 1000.0 * e2e_s, "api": "psacak32_ctx (host pointers, pinned buffers)"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        w = 4 << 20
        t0 = time.perf_counter()
        oracle_lib.psacak32(text[:w].copy())
        dt = time.perf_counter() - t0
        cpu = {"value": w / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "first %d symbols of the workload, one serial oracle build" % w}
    if rank == 0:
        line = {"metric": "suffixes/sec (psacak32 suffix-array build, bit-exact)", "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic", "config": workload_config(args), "e2e": e2e, "roofline": roofline,
                "hbm_gbs_algorithmic_build": algorithmic_build_bytes(trace, 12 * n) / (ms / 1000.0) / 1e9,
                "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches), "verified": verified,
                "levels": [[lv["m"], lv["n_lms"], lv["k"]] for lv in trace],
                "induced_top_level": induced, "zero_schedule": zero}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def dominant_traffic(name, items_per_launch):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (bytes per item measured on a capture, scaled to this launch)."""
    p = os.path.join(ROOT, "profiles", "traffic_per_item.json")
    try:
        with open(p) as f:
            d = json.load(f)
        per_item = d[name]["dram_bytes_per_item"]
        return per_item * items_per_launch
    except Exception:
        return None


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
