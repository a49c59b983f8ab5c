"""Schedule autotuner: chooses the knobs of psacak_schedule by timing builds.

Every schedule builds the same suffix array; the knobs only change speed:

* ``engine``            byte-level induced-scan engine (bucket scan or chain
                        doubling);
* ``tile_items``        items per thread of the bucket scatter and the
                        compactions (8, 12 or 16: the onesweep tile shape);
* ``scan_ctas_per_sm``  CTAs per SM of the grid-stride helper kernels (the
                        block shape of the typing and histogram passes);
* ``batch_chunk_mib``   largest concatenated build of a batch (the chunk size);
* ``finish_below``      recursion strategy: levels shorter than this are
                        sorted directly by prefix doubling; in a batch, texts
                        of at most 8 KiB below it go to one CTA each;
* ``inner_finish_below`` the same cut-off for the reduced strings.

``exhaustive`` times a list of schedules (the fallback of the learned
selector and the yardstick of its regret).  ``coordinate_descent`` searches
a product space one knob at a time -- each knob's values are timed with the
others held at the best so far, for a fixed number of sweeps -- which needs
sum(len(values)) builds per sweep instead of their product; it is what the
batched build uses to pick chunk size and block shape.
"""
import math

BATCH_SPACE = {
    "finish_below": [0, 1 << 13, 1 << 16, 1 << 20, 1 << 22, 1 << 26],
    "batch_chunk_mib": [256, 512, 1024, 3072],
    "tile_items": [8, 12, 16],
    "scan_ctas_per_sm": [2, 4, 8],
    "engine": [1, 2],
    "inner_finish_below": [1 << 30, 1 << 26, 1 << 22],
}
BATCH_ORDER = ["finish_below", "inner_finish_below", "batch_chunk_mib", "tile_items", "scan_ctas_per_sm", "engine"]


def device_timer(build, reps=1):
    """Returns time_fn(schedule) -> device ms (min over `reps` after one
    warm-up build), timed with CUDA events on the current stream."""
    import torch
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def time_fn(sched):
        build(sched)
        best = math.inf
        for _ in range(reps):
            e0.record(stream)
            build(sched)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best
    return time_fn


def exhaustive(time_fn, schedules):
    """Times every schedule; returns (index of the fastest, list of ms)."""
    ms = [time_fn(dict(s)) for s in schedules]
    return min(range(len(ms)), key=ms.__getitem__), ms


def coordinate_descent(time_fn, start, space=None, order=None, sweeps=1):
    """One knob at a time, `sweeps` times over `order`: every value of the
    knob is timed with the other knobs at the best values found so far.
    Returns (best schedule, best ms, table of every timed schedule)."""
    space = BATCH_SPACE if space is None else space
    order = BATCH_ORDER if order is None else order
    best = dict(start)
    seen = {}

    def timed(s):
        key = tuple(sorted(s.items()))
        if key not in seen:
            seen[key] = time_fn(dict(s))
        return seen[key]

    best_ms = timed(best)
    for _ in range(sweeps):
        for knob in order:
            for v in space[knob]:
                cand = dict(best)
                cand[knob] = v
                ms = timed(cand)
                if ms < best_ms:
                    best, best_ms = cand, ms
    table = [{"schedule": dict(k), "ms": v} for k, v in seen.items()]
    return best, best_ms, table
