"""Regenerates the golden fixtures in this folder.

reference_vectors.json
    The known-answer inputs of hucsmn/psacak's own tests: the 'mississippi'
    doc-test (src/lib.rs:12-15, :21-27, :37-42) and the 11-text tables of
    tablecheck_sacak8 / tablecheck_sacak32 (src/psacak8.rs:508-524,
    src/psacak32.rs:826-842), with their suffix arrays computed here by an
    independent pure-Python naive sort (the reference checks these tables
    against saca_tiny, src/common.rs:13-25, which is the same naive sort).

synthetic_traces.json
    For a few seeded synthetic inputs: the oracle's per-level records
    (m, LMS count, name count, reduced-string hash) and a hash of its suffix
    array.  Committed so that the oracle restatement is pinned to fixed
    outputs and GPU tests can compare level by level without re-running the
    oracle on every size.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

TABLES = [
    [0, 0, 0, 0, 0, 0],
    [0, 0, 0, 0, 0, 1],
    [5, 4, 3, 2, 1, 0],
    [3, 4, 5, 2, 0, 1],
    [2, 0, 2, 0, 2, 1, 4, 3],
    [3, 2, 1, 3, 2, 3, 2, 1, 0, 1],
    [2, 1, 4, 1, 1, 4, 1, 3, 1],
    [2, 1, 1, 3, 3, 1, 1, 3, 3, 1, 2, 1],
    [2, 2, 1, 4, 4, 1, 4, 4, 1, 3, 3, 1, 1],
    [6, 8, 9, 5, 2, 4, 3, 0, 0, 7, 1, 2],
    [1, 2, 2, 1, 1, 0, 0, 1, 1, 2, 2, 0, 0, 2, 2, 0, 1, 0, 2, 0, 1, 1, 1, 1, 2, 2, 0, 0, 2, 1, 2, 1, 1, 0,
     2, 1, 2, 2, 0, 2, 1, 1, 2, 2, 2, 1, 2, 0, 0, 1, 2, 0, 0, 0, 1, 2, 2, 2, 1, 1, 1, 1, 2, 0, 2, 1, 1, 1,
     2, 1, 0, 1],
]

SYNTHETIC = [
    # (name, generator, n, seed)
    ("iid_acgt_1m", "iid_acgt", 1 << 20, 11),
    ("genome_2m", "genome", 2 << 20, 12),
    ("zipf32_512k", "zipf32", 1 << 19, 13),
    ("iid_bytes_256k", "iid_bytes", 1 << 18, 14),
    ("markov2_300k", "markov2", 300_001, 15),
]


def naive_sa(seq):
    return sorted(range(len(seq)), key=lambda i: seq[i:])


def make_input(gen, n, seed):
    from psacak_b200 import synth
    if gen == "iid_acgt":
        return synth.iid(n, b"ACGT", seed)
    if gen == "iid_bytes":
        return synth.iid(n, bytes(range(256)), seed)
    if gen == "genome":
        return synth.genome(n, seed)
    if gen == "markov2":
        return synth.markov2(n, seed)
    if gen == "zipf32":
        return synth.zipf32(n, seed=seed)
    raise ValueError(gen)


def main():
    vectors = {
        "mississippi": {"text": "mississippi", "sa": naive_sa(b"mississippi"),
                        "sa_with_sentinel": [11] + naive_sa(b"mississippi")},
        "tables": [{"text": t, "sa": naive_sa(t)} for t in TABLES],
    }
    assert vectors["mississippi"]["sa"] == [10, 7, 4, 1, 0, 9, 8, 6, 3, 5, 2]
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(vectors, f, indent=1)

    import oracle_lib as o
    traces = []
    for name, gen, n, seed in SYNTHETIC:
        t = make_input(gen, n, seed)
        if gen == "zipf32":
            sa, tr = o.psacak32(t, trace=True)
            assert o.check_sa32(t, sa)
        else:
            sa, tr = o.psacak8(t, trace=True)
            assert o.check_sa8(t, sa)
        traces.append({"name": name, "generator": gen, "n": n, "seed": seed,
                       "sa_hash": o.hash_u32(sa), "levels": tr})
        print(name, len(tr), "levels")
    with open(os.path.join(HERE, "synthetic_traces.json"), "w") as f:
        json.dump(traces, f, indent=1)


if __name__ == "__main__":
    main()
