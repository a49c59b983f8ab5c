"""Batched builds (psacak8_batch / psacak8_batch_dev): every text's SA must
equal the oracle's SA of that text alone."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import batch, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def check_all(texts, sas):
    for i, (t, sa) in enumerate(zip(texts, sas)):
        a = np.frombuffer(bytes(t), np.uint8) if isinstance(t, (bytes, bytearray)) else t
        assert (sa == o.psacak8(a)).all(), i


def run_dev(ctx, texts, schedule=None):
    buf, off = batch.pack(texts)
    dt = torch.from_numpy(buf).cuda() if buf.size else torch.zeros(1, dtype=torch.uint8, device="cuda")
    ds = torch.empty(max(buf.size, 1), dtype=torch.int32, device="cuda")
    ctx.psacak8_batch_dev(dt.data_ptr(), off, ds.data_ptr(), torch.cuda.current_stream().cuda_stream, schedule)
    out = ds.cpu().numpy().view(np.uint32)
    return [out[int(off[i]):int(off[i + 1])] for i in range(len(texts))]


def test_small_random_batches(ctx):
    rng = np.random.default_rng(40)
    for trial in range(20):
        k = int(rng.integers(1, 60))
        alpha = int(rng.choice([2, 4, 200]))
        texts = [rng.integers(1, alpha + 1, int(rng.integers(0, 3000))).astype(np.uint8) for _ in range(k)]
        check_all(texts, run_dev(ctx, texts))


def test_batch_with_zero_bytes_and_empty_texts(ctx):
    texts = [b"", b"\x00\x00\x01", b"mississippi", b"", b"\x00", b"ab\x00ab\x00", bytes(range(10)) * 30]
    check_all(texts, run_dev(ctx, texts))


def test_batch_using_every_byte_value(ctx):
    texts = [bytes(range(256)) * 3, b"\x00\xff" * 50, b"abc"]
    check_all(texts, run_dev(ctx, texts))


def test_markov_batch_and_chunking(ctx):
    texts = batch.batch_texts(count=64, lo=1 << 10, hi=256 << 10, seed=41)
    sas = run_dev(ctx, texts)
    check_all(texts, sas)
    sas2 = run_dev(ctx, texts, {"batch_chunk_mib": 1})
    for a, b in zip(sas, sas2):
        assert (a == b).all()


def test_host_batch_api(ctx):
    texts = batch.batch_texts(count=16, lo=100, hi=20000, seed=42)
    check_all(texts, ctx.psacak_batch(texts))
