"""The autotuner's search logic on a fake timer (no GPU): coordinate descent
finds the optimum of a separable cost, times each schedule once, and the
exhaustive search returns the index of the fastest schedule."""
from psacak_b200 import autotune


def _cost(s):
    # separable: each knob has one best value
    best = {"finish_below": 1 << 16, "batch_chunk_mib": 512, "tile_items": 12, "scan_ctas_per_sm": 2, "engine": 1}
    return 10.0 + sum(abs(hash((k, s[k])) % 7) * (0 if s[k] == v else 1) + (0 if s[k] == v else 1)
                      for k, v in best.items())


def test_coordinate_descent_finds_separable_optimum():
    calls = []

    def tf(s):
        calls.append(tuple(sorted(s.items())))
        return _cost(s)

    start = {"finish_below": 0, "batch_chunk_mib": 3072, "tile_items": 8, "scan_ctas_per_sm": 8, "engine": 2}
    best, ms, table = autotune.coordinate_descent(tf, start)
    assert best == {"finish_below": 1 << 16, "batch_chunk_mib": 512, "tile_items": 12, "scan_ctas_per_sm": 2,
                    "engine": 1}
    assert ms == 10.0
    assert len(calls) == len(set(calls)) == len(table)  # every schedule timed once
    assert len(calls) <= 1 + sum(len(v) for v in autotune.BATCH_SPACE.values())


def test_exhaustive_picks_fastest():
    scheds = [{"finish_below": f} for f in (0, 1, 2, 3)]
    i, ms = autotune.exhaustive(lambda s: [5.0, 2.0, 7.0, 3.0][s["finish_below"]], scheds)
    assert i == 1 and ms == [5.0, 2.0, 7.0, 3.0]
