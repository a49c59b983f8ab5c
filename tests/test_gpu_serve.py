"""The serving loop on the GPU, small: Poisson arrivals released by a thread,
two workers serving from host buffers, the selector picking schedules, a
few served suffix arrays compared with the oracle, and the regret report
against exhaustive autotuning."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import selector as sel
from psacak_b200 import serve

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _check(i, text, sa):
    want = o.psacak8(text) if text.dtype == np.uint8 else o.psacak32(text)
    return bool(np.array_equal(sa, want))


def test_serving_loop_small():
    with pk.Context(0) as ctx:
        net = sel.Selector(ctx, k=len(sel.SCHEDULES), seed=1)  # untrained: any pick must still be correct
        res = serve.run(net, count=80, seed=3, load=0.7, workers=2, autotune_sample=6, lo=4 << 10, hi=1 << 20,
                        best_fixed=0, probe=40, check=_check)
    assert res["requests"] == 80 and sum(res["requests_per_worker"]) == 80
    assert res["checked_against_oracle"]["requests"] > 0
    assert res["checked_against_oracle"]["equal"] == res["checked_against_oracle"]["requests"]
    assert 0 < res["p50_latency_ms"] <= res["p99_latency_ms"]
    assert res["throughput_suffixes_per_s"] > 0
    for k in ("regret_selector", "regret_best_fixed", "regret_library_default"):
        assert res[k]["mean"] >= 0.0
    assert sum(res["schedule_histogram"].values()) == 80


def test_serving_without_a_model_uses_the_library_default():
    res = serve.run(None, count=20, seed=4, load=0.5, workers=2, autotune_sample=0, lo=4 << 10, hi=256 << 10,
                    probe=10, check=_check)
    assert res["checked_against_oracle"]["equal"] == res["checked_against_oracle"]["requests"]
    assert sum(res["schedule_histogram"].values()) == 0  # no picks: NULL schedule
