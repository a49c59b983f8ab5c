"""Failure detection in the forms a shared GPU allows: no test faults, traps
or hangs the device.

* A bounded device wait that runs out: the single-pass look-back scan of
  every build, launched without its first tile, waits on status words that
  nothing publishes; with a short poll limit the waits give up, the call
  returns PSACAK_ETIMEOUT, and the same context then builds correct suffix
  arrays.
* An allocation failure: a workspace cap on the context makes a build's
  allocation fail with PSACAK_ENOMEM; without the cap the context rebuilds.
* A cancelled batch: psacak_cancel ends the build with PSACAK_ECANCELED,
  pending or from another thread; the context stays usable.

The reference panics on misuse and has nothing to time out or cancel
(src/lib.rs:65, :78-79); these statuses replace its panics at the C ABI.
"""
import threading
import time

import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import batch as pb
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _build_and_compare(ctx, text):
    sa = ctx.psacak(text)
    assert np.array_equal(sa, o.psacak8(text))


def test_look_back_wait_runs_out_then_context_recovers():
    with pk.Context(0) as ctx:
        st = pk.Stages(ctx)
        n = 64 * 4096 + 17
        x = np.random.default_rng(1).integers(0, 1000, n, dtype=np.uint32)
        d_in = torch.from_numpy(x.view(np.int32)).cuda()
        d_out = torch.zeros(n, dtype=torch.int32, device="cuda")
        st.set_limits(spin_limit=2000)
        t0 = time.time()
        rc = st.stalled_scan(d_in.data_ptr(), d_out.data_ptr(), n)
        assert rc == pk.PSACAK_ETIMEOUT, rc
        assert b"wait ran out" in pk.lib().psacak_last_error_string()
        assert time.time() - t0 < 30
        # a second stalled launch times out again (fresh epoch, stale words unread)
        assert st.stalled_scan(d_in.data_ptr(), d_out.data_ptr(), n) == pk.PSACAK_ETIMEOUT
        # back to the compiled limits: the same context scans and builds correctly
        st.set_limits(spin_limit=0)
        st.exclusive_sum(d_in.data_ptr(), d_out.data_ptr(), n)
        want = np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]).astype(np.uint32)
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want)
        _build_and_compare(ctx, synth.genome(1 << 20, seed=41))


def test_short_wait_limit_does_not_disturb_a_normal_build():
    # a limit well above what the predecessors need still builds correctly
    with pk.Context(0) as ctx:
        pk.Stages(ctx).set_limits(spin_limit=1 << 20)
        _build_and_compare(ctx, synth.genome(2 << 20, seed=42))
        _build_and_compare(ctx, synth.iid(1 << 20, b"ACGT", seed=43))


def test_stalled_scan_rejects_one_tile():
    with pk.Context(0) as ctx:
        d = torch.zeros(4096, dtype=torch.int32, device="cuda")
        assert pk.Stages(ctx).stalled_scan(d.data_ptr(), d.data_ptr(), 4096) == pk.PSACAK_EINVAL


@pytest.mark.parametrize("cap", [1 << 16, 8 << 20])
def test_allocation_failure_is_enomem_then_clean_rebuild(cap):
    text = synth.genome(4 << 20, seed=44)
    n = text.size
    with pk.Context(0) as ctx:
        st = pk.Stages(ctx)
        dt = torch.from_numpy(text).cuda()
        ds = torch.zeros(n, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        st.set_limits(workspace_cap=cap)
        with pytest.raises(pk.PsacakError) as e:
            ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream)
        assert e.value.code == pk.PSACAK_ENOMEM
        assert "workspace cap" in str(e.value)
        with pytest.raises(pk.PsacakError) as e:
            ctx.psacak32_dev(torch.from_numpy(text.astype(np.uint32).view(np.int32)).cuda().data_ptr(), n,
                             ds.data_ptr(), stream)
        assert e.value.code == pk.PSACAK_ENOMEM
        st.set_limits(workspace_cap=0)
        ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream)
        torch.cuda.synchronize()
        assert np.array_equal(ds.cpu().numpy().view(np.uint32), o.psacak8(text))
        _build_and_compare(ctx, synth.genome(1 << 20, seed=45))


def _batch(count, seed, hi=1 << 20):
    return pb.batch_texts(count=count, lo=1 << 10, hi=hi, seed=seed)


def test_pending_cancel_ends_the_next_batch():
    texts = _batch(48, 46)
    with pk.Context(0) as ctx:
        ctx.cancel()
        with pytest.raises(pk.PsacakError) as e:
            ctx.psacak_batch(texts)
        assert e.value.code == pk.PSACAK_ECANCELED
        # the request was consumed: the next batch runs to the end
        sas = ctx.psacak_batch(texts)
        for t, sa in zip(texts, sas):
            assert np.array_equal(sa, o.psacak8(t))
        # a single build is cancelled the same way
        ctx.cancel()
        with pytest.raises(pk.PsacakError) as e:
            ctx.psacak(texts[0])
        assert e.value.code == pk.PSACAK_ECANCELED
        _build_and_compare(ctx, texts[1])


def test_cancel_from_another_thread():
    texts = _batch(160, 47, hi=4 << 20)
    with pk.Context(0) as ctx:
        ctx.psacak_batch(texts[:4])  # warm the workspace
        outcome = {}

        def run():
            try:
                ctx.psacak_batch(texts, schedule={"batch_chunk_mib": 8})
                outcome["rc"] = pk.PSACAK_OK
            except pk.PsacakError as ex:
                outcome["rc"] = ex.code

        th = threading.Thread(target=run)
        th.start()
        time.sleep(0.05)
        ctx.cancel()
        th.join(120)
        assert not th.is_alive()
        assert outcome["rc"] in (pk.PSACAK_OK, pk.PSACAK_ECANCELED)
        if outcome["rc"] == pk.PSACAK_OK:
            # the request came after the batch's last checkpoint: it ends
            # the next call instead
            with pytest.raises(pk.PsacakError) as e:
                ctx.psacak(b"xyz")
            assert e.value.code == pk.PSACAK_ECANCELED
        sas = ctx.psacak_batch(texts[:24])
        for t, sa in zip(texts[:24], sas):
            assert np.array_equal(sa, o.psacak8(t))
