"""The benchmark workloads at their full sizes, built on the GPU and compared
with the oracle's results for the same inputs (fixtures written by
tests/golden/make_fullsize.py: the oracle's suffix array of each input,
reduced to a hash, and its per-level records).

* psacak8 on the 1 GiB genome-like text (seed 2): the device-pointer call
  the bench times and the host-pointer call (pageable output, the Rust
  `psacak_inplace` shape); SA hash and every level's (m, LMS count, name
  count, reduced-string hash).
* psacak32 on 2^28 Zipf symbols over 2^20 with planted repeats (seed 2):
  the default schedule (prefix doubling from the text), induced sorting at
  the top level with prefix doubling below, and the zero schedule whose
  recursion goes all the way down as the oracle's does (trace compared
  level by level).
* the 4096-text batch (seed 2): every text's SA hash, with the library's
  default schedule and with a chunked schedule of the kind the autotuner
  picks.

Hashes are the oracle's hash_u32 of the arrays copied back to the host.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import batch as pb
from psacak_b200 import synth

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
torch = pytest.importorskip("torch")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def _u32(t):
    return t.cpu().numpy().view(np.uint32)


# PSACAK_DEFAULT_FINISH_BELOW (bytes) or _BELOW32 (integers), PSACAK_DEFAULT_INNER_FINISH_BELOW
DEFAULT_FINISH8 = (1 << 24, 1 << 30)
DEFAULT_FINISH32 = (1 << 30, 1 << 30)


def _levels_match(got, want, finish):
    """The levels a build recursed through are the oracle's; from the first
    level shorter than its cut-off on (finish[0] for the input, finish[1]
    for the reduced strings), the build sorted directly by prefix doubling
    (one record, no LMS count) where the oracle recursed further."""
    assert len(got) <= len(want)
    for i, (lv, w) in enumerate(zip(got, want)):
        cut = finish[0] if i == 0 else finish[1]
        if cut and lv["m"] < cut and w["n_lms"] > 0:
            assert lv["m"] == w["m"] and lv["n_lms"] == 0 and i == len(got) - 1
            return
        assert lv == w
    assert len(got) == len(want)


def test_genome_1gib_matches_oracle(ctx):
    fx = load("fullsize_genome1g.json")
    n = fx["n"]
    text = synth.genome(n, seed=fx["seed"])
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(text).cuda()
    ds = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream, None)
    torch.cuda.synchronize()
    _levels_match(ctx.trace(), fx["levels"], DEFAULT_FINISH8)
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    assert ctx.check_sa8_dev(dt.data_ptr(), n, ds.data_ptr(), stream)
    # induced sorting down to 64 Mi symbols, the old default's shape
    ds.zero_()
    ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream, {"engine": 1, "tile_items": 16,
                                                             "finish_below": 1 << 26})
    torch.cuda.synchronize()
    _levels_match(ctx.trace(), fx["levels"], (1 << 26, 1 << 26))
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    # the zero schedule recurses all the way down, as the oracle does
    ds.zero_()
    ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream, {"engine": pk.ENGINE_BUCKET})
    torch.cuda.synchronize()
    assert ctx.trace() == fx["levels"]
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    del ds, dt
    torch.cuda.empty_cache()
    # host pointers, pageable output: the drop-in for psacak_inplace
    sa = ctx.psacak(text)
    assert o.hash_u32(sa) == fx["sa_hash"]


def test_zipf32_256m_matches_oracle(ctx):
    fx = load("fullsize_zipf32_256m.json")
    n = fx["n"]
    text = synth.zipf32(n, alphabet=1 << 20, s=1.1, repeat_frac=0.10, rep_min=1000, rep_max=100000,
                        seed=fx["seed"])
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(text.view(np.int32)).cuda()
    ds = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.psacak32_dev(dt.data_ptr(), n, ds.data_ptr(), stream, None)
    torch.cuda.synchronize()
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    # the levels the default schedule recursed through are the oracle's
    _levels_match(ctx.trace(), fx["levels"], DEFAULT_FINISH32)
    # induced sorting at the top level, prefix doubling from the first reduced string on
    ds.zero_()
    ctx.psacak32_dev(dt.data_ptr(), n, ds.data_ptr(), stream, {"tile_items": 16, "finish_below": 1 << 26,
                                                             "inner_finish_below": 1 << 30})
    torch.cuda.synchronize()
    _levels_match(ctx.trace(), fx["levels"], (1 << 26, 1 << 30))
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    ds.zero_()
    ctx.psacak32_dev(dt.data_ptr(), n, ds.data_ptr(), stream, {})  # zero schedule: no finisher
    torch.cuda.synchronize()
    assert ctx.trace() == fx["levels"]
    assert o.hash_u32(_u32(ds)) == fx["sa_hash"]
    assert ctx.check_sa32_dev(dt.data_ptr(), n, ds.data_ptr(), stream)


@pytest.mark.parametrize("schedule", [None, {"engine": 1, "tile_items": 12, "scan_ctas_per_sm": 2,
                                             "batch_chunk_mib": 256, "finish_below": 1 << 13}])
def test_batch4096_matches_oracle(ctx, schedule):
    fx = load("fullsize_batch4096.json")
    texts = pb.batch_texts(count=fx["count"], seed=fx["seed"])
    buf, off = pb.pack(texts)
    assert int(off[-1]) == fx["total_bytes"]
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(buf).cuda()
    ds = torch.empty(buf.size, dtype=torch.int32, device="cuda")
    ctx.psacak8_batch_dev(dt.data_ptr(), off, ds.data_ptr(), stream, schedule)
    torch.cuda.synchronize()
    sa = _u32(ds)
    bad = [i for i in range(len(texts))
           if "%016x" % o.hash_u32(sa[int(off[i]):int(off[i + 1])]) != fx["sa_hashes"][i]]
    assert not bad, bad[:10]
