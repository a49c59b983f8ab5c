"""Learned schedule selection for psacak_b200.

* ``SCHEDULES`` -- the candidate schedules (engine of the byte level x scatter
  tile size x recursion strategy: levels shorter than ``finish_below`` --
  level 0 included -- are sorted directly by prefix doubling).  Every one
  builds the same suffix array.
* ``features`` -- 16 text statistics computed on the GPU (psacak_text_stats).
* ``autotune`` -- exhaustive search: times every schedule on a text.  It is
  the fallback when no trained model is available and the yardstick for the
  model's picks (regret = picked time / best time - 1).
* ``Selector`` -- fp32 MLP 16 -> 64 -> 64 -> K predicting log2(ms) of every
  schedule; trained on the GPU by the library's own forward / backward / Adam
  kernels (include/psacak_b200_select.h); inference is one kernel launch.
"""
import ctypes
import json
import math
import os

import numpy as np

from . import lib, _raise, _sched_ptr, ENGINE_BUCKET, ENGINE_DOUBLING

NF = 16
NH = 64

# Recursion strategy is the knob whose best value depends on the text: prefix
# doubling needs log2(longest repeat) rounds over every unresolved suffix, so
# it wins on repeat-poor texts of any length and loses on repetitive ones,
# where induced sorting and recursion win.  0 = never, ALWAYS = the whole
# text is sorted by prefix doubling.
ALWAYS = 0xFFFFFFFF
FINISH_GRID = [0, 1 << 16, 1 << 18, 1 << 20, 1 << 22, 1 << 24, 1 << 26, ALWAYS]
# The reduced strings of every schedule use the library's inner cut-off
# (1 Gi symbols): prefix doubling from the first reduced string on.
INNER_FINISH = 1 << 30
SCHEDULES = [
    {"engine": ENGINE_BUCKET, "inner_engine": ENGINE_DOUBLING, "tile_items": t, "finish_below": f,
     "inner_finish_below": INNER_FINISH}
    for t in (8, 16) for f in FINISH_GRID
]


def library_default(width):
    """The schedule a NULL psacak_schedule stands for (include/psacak_b200.h):
    the cut-off depends on the symbol width."""
    return {"engine": ENGINE_BUCKET, "inner_engine": ENGINE_DOUBLING, "tile_items": 16,
            "finish_below": 1 << 24 if width == 1 else 1 << 30, "inner_finish_below": INNER_FINISH}


def _bind():
    L = lib()
    if getattr(L, "_sel_bound", False):
        return L
    p, u64, u32, i32, f32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    L.psacak_sel_param_count.argtypes = [u32]
    L.psacak_sel_param_count.restype = u64
    L.psacak_text_stats.argtypes = [p, p, u64, i32, p]
    L.psacak_mlp_forward.argtypes = [p, p, p, p, p, p, u32, u32]
    L.psacak_mlp_backward.argtypes = [p, p, p, p, p, p, p, p, p, u32, u32, f32, ctypes.POINTER(f32)]
    L.psacak_mlp_adam.argtypes = [p, p, p, p, p, u64, f32, f32, f32, f32, u32]
    L.psacak_select_schedule.argtypes = [p, p, u32, p, ctypes.POINTER(u32), p]
    L.psacak_gen_iid_dev.argtypes = [p, p, u64, i32, p, u32, u64, p]
    for nm in ("psacak_text_stats", "psacak_mlp_forward", "psacak_mlp_backward", "psacak_mlp_adam",
               "psacak_select_schedule", "psacak_gen_iid_dev"):
        getattr(L, nm).restype = i32
    L._sel_bound = True
    return L


def param_count(k):
    return int(_bind().psacak_sel_param_count(k))


def features(ctx, d_text, n, width):
    """16 statistics of a device-resident text (width 1 = bytes, 4 = u32)."""
    out = np.zeros(NF, dtype=np.float32)
    _raise(_bind().psacak_text_stats(ctx.handle, ctypes.c_void_p(d_text), n, width,
                                     out.ctypes.data_as(ctypes.c_void_p)))
    return out


def gen_iid_dev(ctx, d_out, n, width, alphabet, seed, stream=0):
    """Fills d_out with an i.i.d. text (bytes from `alphabet`, or u32 symbols
    uniform on [0, alphabet) when width == 4)."""
    if width == 1:
        a = np.frombuffer(bytes(alphabet), np.uint8).copy()
        _raise(_bind().psacak_gen_iid_dev(ctx.handle, ctypes.c_void_p(d_out), n, 1,
                                          a.ctypes.data_as(ctypes.c_void_p), a.size, seed, ctypes.c_void_p(stream)))
    else:
        _raise(_bind().psacak_gen_iid_dev(ctx.handle, ctypes.c_void_p(d_out), n, 4, None, int(alphabet), seed,
                                          ctypes.c_void_p(stream)))


def build(ctx, d_text, n, width, d_sa, stream, schedule):
    if width == 1:
        ctx.psacak8_dev(d_text, n, d_sa, stream, schedule)
    else:
        ctx.psacak32_dev(d_text, n, d_sa, stream, schedule)


def autotune(ctx, d_text, n, width, d_sa, reps=2, schedules=SCHEDULES):
    """Device milliseconds of every schedule on one text (min over reps,
    after one warm-up build); a None schedule is the library default."""
    import torch
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    times = np.zeros(len(schedules), dtype=np.float64)
    for k, sc in enumerate(schedules):
        build(ctx, d_text, n, width, d_sa, stream.cuda_stream, sc)
        best = math.inf
        for _ in range(reps):
            e0.record(stream)
            build(ctx, d_text, n, width, d_sa, stream.cuda_stream, sc)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        times[k] = best
    return times


class Selector:
    """fp32 MLP predicting log2(ms) per schedule; params live on the GPU."""

    def __init__(self, ctx, k=len(SCHEDULES), seed=0, params=None):
        import torch
        self.ctx = ctx
        self.k = k
        self.np = param_count(k)
        if params is None:
            g = np.random.default_rng(seed)
            p = np.zeros(self.np, dtype=np.float32)
            o = 0
            for fan_in, fan_out in ((NF, NH), (NH, NH), (NH, k)):
                w = (g.standard_normal((fan_in, fan_out)) * math.sqrt(2.0 / fan_in)).astype(np.float32)
                p[o:o + w.size] = w.ravel()
                o += w.size + fan_out  # biases stay 0
            params = p
        self.params = torch.from_numpy(np.asarray(params, dtype=np.float32).copy()).cuda()

    def bind(self, ctx):
        """The same network (parameters shared, not copied) driven through
        another context, e.g. one per serving thread."""
        other = object.__new__(Selector)
        other.ctx, other.k, other.np, other.params = ctx, self.k, self.np, self.params
        return other

    def _ptr(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def forward(self, X):
        import torch
        X = torch.as_tensor(np.asarray(X, np.float32)).cuda().contiguous()
        B = X.shape[0]
        Y = torch.empty((B, self.k), dtype=torch.float32, device="cuda")
        H1 = torch.empty((B, NH), dtype=torch.float32, device="cuda")
        H2 = torch.empty((B, NH), dtype=torch.float32, device="cuda")
        _raise(_bind().psacak_mlp_forward(self.ctx.handle, self._ptr(self.params), self._ptr(X), self._ptr(Y),
                                          self._ptr(H1), self._ptr(H2), B, self.k))
        return X, Y, H1, H2

    def gradients(self, X, T, M):
        """(loss, grads) of the masked MSE on one batch (device tensors)."""
        import torch
        Xd, Y, H1, H2 = self.forward(X)
        Td = torch.as_tensor(np.asarray(T, np.float32)).cuda().contiguous()
        Md = torch.as_tensor(np.asarray(M, np.float32)).cuda().contiguous()
        G = torch.empty(self.np, dtype=torch.float32, device="cuda")
        loss = ctypes.c_float(0)
        _raise(_bind().psacak_mlp_backward(self.ctx.handle, self._ptr(self.params), self._ptr(Xd), self._ptr(H1),
                                           self._ptr(H2), self._ptr(Y), self._ptr(Td), self._ptr(Md), self._ptr(G),
                                           Xd.shape[0], self.k, float(Md.sum().item()), ctypes.byref(loss)))
        return loss.value, G

    def train(self, X, T, M, epochs=2000, lr=3e-3, log_every=0):
        """Full-batch Adam on the GPU; returns the loss history."""
        import torch
        m1 = torch.zeros(self.np, dtype=torch.float32, device="cuda")
        m2 = torch.zeros(self.np, dtype=torch.float32, device="cuda")
        hist = []
        for step in range(1, epochs + 1):
            loss, G = self.gradients(X, T, M)
            _raise(_bind().psacak_mlp_adam(self.ctx.handle, self._ptr(self.params), self._ptr(G), self._ptr(m1),
                                           self._ptr(m2), self.np, lr, 0.9, 0.999, 1e-8, step))
            hist.append(loss)
            if log_every and step % log_every == 0:
                print("step %d loss %.5f" % (step, loss), flush=True)
        return hist

    def predict(self, feats):
        """(index of the fastest predicted schedule, predictions) via the
        inference kernel."""
        f = np.ascontiguousarray(feats, dtype=np.float32)
        pred = np.zeros(self.k, dtype=np.float32)
        choice = ctypes.c_uint32(0)
        _raise(_bind().psacak_select_schedule(self.ctx.handle, self._ptr(self.params), self.k,
                                              f.ctypes.data_as(ctypes.c_void_p), ctypes.byref(choice),
                                              pred.ctypes.data_as(ctypes.c_void_p)))
        return int(choice.value), pred

    def save(self, path, meta=None):
        np.savez(path, params=self.params.cpu().numpy(), k=self.k,
                 meta=json.dumps(meta or {}), schedules=json.dumps(SCHEDULES))

    @classmethod
    def load(cls, ctx, path):
        """The saved network, or None when it was trained for another
        schedule list than SCHEDULES (its outputs would not index it)."""
        d = np.load(path, allow_pickle=False)
        if "schedules" not in d.files or json.loads(str(d["schedules"])) != SCHEDULES:
            return None
        return cls(ctx, k=int(d["k"]), params=d["params"])


def targets(times):
    """log2(ms) targets and masks from autotune results (rows of times)."""
    T = np.log2(np.maximum(np.asarray(times, np.float64), 1e-3)).astype(np.float32)
    return T, np.ones_like(T)


# -- CPU fp32 reference of the network (for gradient checks) ------------------
def ref_forward(p, X, k):
    X = np.asarray(X, np.float32)
    o = 0
    W1 = p[o:o + NF * NH].reshape(NF, NH); o += NF * NH
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    W3 = p[o:o + NH * k].reshape(NH, k); o += NH * k
    b3 = p[o:o + k]
    H1 = np.maximum(X @ W1 + b1, 0).astype(np.float32)
    H2 = np.maximum(H1 @ W2 + b2, 0).astype(np.float32)
    Y = (H2 @ W3 + b3).astype(np.float32)
    return Y, H1, H2, (W1, W2, W3)


def ref_gradients(p, X, T, M, k):
    X = np.asarray(X, np.float32)
    Y, H1, H2, (W1, W2, W3) = ref_forward(p, X, k)
    s = float(np.sum(M))
    E = (Y - T) * M
    loss = float(np.sum(E * (Y - T)) / s)
    dY = (2.0 * E / s).astype(np.float32)
    dW3 = H2.T @ dY
    db3 = dY.sum(0)
    dH2 = (dY @ W3.T) * (H2 > 0)
    dW2 = H1.T @ dH2
    db2 = dH2.sum(0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    dW1 = X.T @ dH1
    db1 = dH1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3]).astype(np.float32)
    return loss, g
