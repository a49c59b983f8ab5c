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
          path) on a bounded window of the same text.

`--impl reference` times that CPU oracle instead, on the host cores.
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
    ap.add_argument("--cpu-window", type=int, default=16 << 20, help="bytes per CPU-oracle sample")
    ap.add_argument("--engine", type=int, default=0, help="psacak_schedule.engine (0 = auto)")
    ap.add_argument("--profile-json", default="", help="also write per-kernel stats here")
    ap.add_argument("--single-build", action="store_true",
                    help="build the workload once and exit (for ncu launch lists)")
    return ap.parse_args()


def workload_config(args):
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
def _oracle_window(window_bytes):
    """Oracle build of one window (runs in a spawned worker); returns the
    window length and the build's own wall time."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    text = np.frombuffer(window_bytes, dtype=np.uint8)
    t0 = time.perf_counter()
    sa = oracle_lib.psacak8(text)
    dt = time.perf_counter() - t0
    return int(sa.size), dt


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
    """CPU oracle on the host cores: one independent window build per core."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    from psacak_b200 import synth
    cores = os.cpu_count() or 1
    window = min(args.cpu_window, args.bytes)
    # the first cores x window bytes of the workload text, one window per core
    head = synth.genome(min(cores * window, args.bytes), seed=args.seed)
    jobs = [head[(i * window) % max(head.size - window + 1, 1):][:window].tobytes() for i in range(cores)]
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(cores) as pool:
        for step in range(args.warmup + args.steps):
            res = pool.map(_oracle_window, jobs, chunksize=1)
            if step >= args.warmup:
                # the builds run concurrently: the step lasts as long as the slowest
                times.append((sum(r[0] for r in res), max(r[1] for r in res)))
    total = sum(s for s, _ in times)
    secs = sum(d for _, d in times)
    value = total / secs
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * secs / max(len(times), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "per step, %d independent oracle builds (one per core) of %d-byte windows of "
                                   "the workload text; C++ restatement of the reference's serial path (the Rust "
                                   "crate is unbuildable on this image)" % (cores, window)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# -- GPU arm -------------------------------------------------------------------
def run_b200(args):
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

    text = make_text(args)
    n = text.size
    ctx = pk.Context(local)
    sched = {"engine": args.engine}
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
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        build()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    launches = (ctx.kernel_launches() - l0) // max(args.steps, 1)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1000.0)

    # roofline of the dominant kernel: one more build with the event profiler
    ctx.profile_reset()
    ctx.profile(True)
    build()
    torch.cuda.synchronize(dev)
    ctx.profile(False)
    stats = ctx.profile_stats()
    total_ms = sum(s["ms"] for s in stats)
    dom = max((s for s in stats if s["bytes"] > 0), key=lambda s: s["ms"])
    peak, peak_kind = measured_peak_hbm()
    achieved = dom["bytes"] / (dom["ms"] / 1000.0) / 1e9
    traffic = dominant_traffic(dom["name"], dom["items"] / max(dom["launches"], 1))
    roofline = {"bound": "hbm", "kernel": dom["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "launches": dom["launches"],
                "algorithmic_bytes_per_launch": dom["bytes"] / max(dom["launches"], 1),
                "avg_launch_ms": dom["ms"] / max(dom["launches"], 1),
                "share_of_profiled_time": dom["ms"] / total_ms if total_ms else None}
    build_bytes = algorithmic_build_bytes(trace)
    build_gbs = build_bytes / (ms / 1000.0) / 1e9
    if args.profile_json and rank == 0:
        with open(args.profile_json, "w") as f:
            json.dump({"stats": stats, "trace": trace, "ms_per_step": ms}, f, indent=1)

    # end to end through the host-pointer C ABI
    e2e = None
    if not args.no_e2e:
        h_text = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        h_text.numpy()[:] = text
        h_sa = torch.empty(n, dtype=torch.int32, pin_memory=True)
        ht, hs = h_text.numpy(), h_sa.numpy().view(np.uint32)
        lib = pk.lib()
        import ctypes
        times = []
        for i in range(args.e2e_steps + 1):
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            rc = lib.psacak8_ctx(ctx.handle, ctypes.c_void_p(ht.ctypes.data), n, ctypes.c_void_p(hs.ctypes.data),
                                 pk._sched_ptr(sched))
            dt = time.perf_counter() - t0
            if rc != 0:
                pk._raise(rc)
            if i > 0:
                times.append(dt)
        e2e_s = float(np.mean(times))
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n, "d2h_bytes_per_step": 4 * n,
               "ms_per_step": 1000.0 * e2e_s, "api": "psacak8_ctx (host pointers, pinned buffers)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_single(text, min(args.cpu_window, n))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic", "config": workload_config(args),
            "e2e": e2e, "roofline": roofline,
            "hbm_gbs_algorithmic_build": build_gbs,
            "build_algorithmic_bytes": build_bytes,
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "verified": verified, "levels": [[lv["m"], lv["n_lms"], lv["k"]] for lv in trace],
        }
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
