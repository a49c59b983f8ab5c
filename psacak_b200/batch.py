"""Host-side helpers for batched builds: packing and multi-GPU sharding.

A batch of independent texts is built with one psacak8_batch_dev call per
GPU.  Across GPUs the texts are split with longest-processing-time-first
(each text to the rank with the smallest total so far, longest texts first):
no data-path collective is needed, every rank writes its own texts' SAs.
"""
import heapq

import numpy as np


def pack(texts):
    """Packs byte texts back to back; returns (uint8 buffer, uint64 offsets)."""
    lens = np.array([len(t) for t in texts], dtype=np.uint64)
    off = np.zeros(len(texts) + 1, dtype=np.uint64)
    np.cumsum(lens, out=off[1:])
    buf = np.empty(int(off[-1]), dtype=np.uint8)
    for i, t in enumerate(texts):
        buf[int(off[i]):int(off[i + 1])] = np.frombuffer(bytes(t), np.uint8) if isinstance(t, (bytes, bytearray)) else t
    return buf, off


def shard_lpt(lengths, world):
    """Assigns text indices to `world` ranks, longest first onto the least
    loaded rank.  Returns a list of sorted index lists, one per rank."""
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(lengths[i]), r))
    return [sorted(x) for x in out]


def batch_texts(count=4096, lo=1 << 10, hi=4 << 20, seed=4):
    """The batched workload: `count` ACGT order-2 Markov texts with lengths
    log-uniform on [lo, hi], text i seeded by hash(seed, i)."""
    from . import synth
    lens = synth.loguniform(count, lo, hi, seed)
    return [synth.markov2(int(n), synth.hash2(seed, i)) for i, n in enumerate(lens)]
