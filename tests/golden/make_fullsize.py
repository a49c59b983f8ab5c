"""Regenerates the full-size golden fixtures: the oracle's suffix arrays of the
benchmark workloads at their full sizes, reduced to hashes.

fullsize_genome1g.json
    psacak8 on the 1 GiB genome-like text (synth.genome(2^30, seed=2)):
    hash of the suffix array and the per-level records (m, LMS count, name
    count, reduced-string hash).
fullsize_zipf32_256m.json
    psacak32 on 2^28 u32 symbols, Zipf(1.1) over 2^20 with 10% planted
    repeats of 1K..100K (synth.zipf32(..., seed=2)): the same records.
fullsize_batch4096.json
    The 4096-text batch (batch.batch_texts(4096, seed=2)): one suffix-array
    hash per text.

The hashes are the oracle's hash_u32 (sum over i of mix64((i << 32) ^ v[i])).
Every oracle result is also put through the oracle's O(n) suffix-array check
before it is written.  The oracle is a restatement of the reference's serial
path, so this takes a few minutes of CPU per workload.

Run from the repository root:
    python tests/golden/make_fullsize.py [genome1g|zipf32_256m|batch4096 ...]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

GENOME_N = 1 << 30
ZIPF_N = 1 << 28
BATCH_COUNT = 4096
SEED = 2


def genome1g():
    import oracle_lib as o
    from psacak_b200 import synth
    text = synth.genome(GENOME_N, seed=SEED)
    sa, tr = o.psacak8(text, trace=True)
    assert o.check_sa8(text, sa)
    return {"workload": "psacak8, synth.genome(2^30, seed=2)", "n": GENOME_N, "seed": SEED,
            "sa_hash": o.hash_u32(sa), "levels": tr}


def zipf32_256m():
    import oracle_lib as o
    from psacak_b200 import synth
    text = synth.zipf32(ZIPF_N, alphabet=1 << 20, s=1.1, repeat_frac=0.10, rep_min=1000, rep_max=100000, seed=SEED)
    sa, tr = o.psacak32(text, trace=True)
    assert o.check_sa32(text, sa)
    return {"workload": "psacak32, synth.zipf32(2^28, alphabet 2^20, s 1.1, 10% repeats 1K..100K, seed=2)",
            "n": ZIPF_N, "seed": SEED, "sa_hash": o.hash_u32(sa), "levels": tr}


def batch4096():
    import oracle_lib as o
    from psacak_b200 import batch
    texts = batch.batch_texts(count=BATCH_COUNT, seed=SEED)
    hashes = []
    for t in texts:
        sa = o.psacak8(t)
        assert o.check_sa8(t, sa)
        hashes.append("%016x" % o.hash_u32(sa))
    return {"workload": "psacak8 per text, batch.batch_texts(4096, seed=2)", "count": BATCH_COUNT, "seed": SEED,
            "total_bytes": int(sum(len(t) for t in texts)), "sa_hashes": hashes}


JOBS = {"genome1g": genome1g, "zipf32_256m": zipf32_256m, "batch4096": batch4096}


def main(names):
    for name in names or JOBS:
        t0 = time.time()
        rec = JOBS[name]()
        with open(os.path.join(HERE, "fullsize_%s.json" % name), "w") as f:
            json.dump(rec, f, indent=1)
        print(name, "%.0f s" % (time.time() - t0), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
