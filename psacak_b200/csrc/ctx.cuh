// ctx.cuh -- builder context: device, stream, stream-ordered allocations,
// scratch for the primitives, the per-level trace.
#pragma once

#include <stdio.h>
#include <time.h>

#include <atomic>
#include <mutex>
#include <utility>
#include <vector>

#include "hostio.cuh"
#include "level.cuh"
#include "radix.cuh"

struct psacak_ctx;

namespace psk {

struct HostStage;  // staging ring and host copy threads (hostio.cu)

struct Ctx {
    Device dev;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;  // stream of the current call
    cudaMemPool_t pool = nullptr;
    uint32_t *h_pinned = nullptr;   // small pinned, mapped buffer for scalar read-backs
    uint32_t *m_pinned = nullptr;   // its device view
    uint32_t *d_hist = nullptr;     // 256 * RADIX_MAX_CTAS radix histograms
    uint32_t *d_scalars = nullptr;  // 64 device scalars
    uint32_t *d_err = nullptr;      // device error word, then the wait-limit override (common.cuh)
    uint32_t *h_hist = nullptr;     // pinned, mapped copy of the radix digit counts
    uint32_t *m_hist = nullptr;     // its device view
    OnesweepScratch os;             // look-back status words of the onesweep kernels
    ScanScratch ss;                 // look-back flags and values of the single-pass scans
    uint32_t scan_ctas = 0;         // CTAs of the grid-stride helper kernels
    uint32_t radix_ctas = 0;        // CTAs of the radix passes
    psacak_schedule sched{};
    // When set, level 0 stops after building its reduced string and copies
    // it here (used by psacak_debug_reduced8).
    uint32_t *debug_red = nullptr;
    uint64_t debug_cap = 0, debug_n1 = 0, debug_k = 0;
    std::vector<psacak_level_info> trace;
    // Reduced-string hashes of the trace are computed into d_hashes (one
    // u64 per level, up to HASH_SLOTS) and read back once, when the build
    // has finished (resolve_trace), instead of a read-back per level.
    static constexpr uint32_t HASH_SLOTS = 64;
    unsigned long long *d_hashes = nullptr;
    std::vector<std::pair<size_t, uint32_t>> pending_hash;  // (trace index, slot)
    bool profiling = false;
    bool stage_timing = false;  // PSACAK_STAGE_TIMES=1: sync + print wall time per stage
    double stage_t0 = 0;
    Profiler prof;
    unsigned long long *d_induced = nullptr;  // entries scattered by the bucket scans
    std::mutex mu;
    // Most workspace bytes a build may hold at once (0 = no cap); a larger
    // request fails with PSACAK_ENOMEM as a failed allocation would.
    uint64_t ws_cap = 0;
    // Set by psacak_cancel from any thread; the build polls it at its
    // checkpoints (recursion levels, doubling rounds, batch chunks).
    std::atomic<uint32_t> cancel_req{0};
    // Checkpoint of a build: consumes a pending cancellation request, lets
    // the work already queued finish (so no buffer is recycled under a
    // running kernel) and ends the build with PSACAK_ECANCELED.
    status_t checkpoint() {
        if (!cancel_req.load(std::memory_order_relaxed) || !cancel_req.exchange(0)) return PSACAK_OK;
        cudaStreamSynchronize(stream);
        return set_error(PSACAK_ECANCELED, "the build was cancelled");
    }

    // Host destination of the final suffix array, set by host-pointer calls
    // whose output buffer is pinned: the level-0 bucket scans send each
    // bucket part to it as soon as that part is final (on copy_stream, after
    // an event on the build stream), so the copy overlaps the rest of the
    // build.  sink_done tells the caller that every slot was sent.
    uint32_t *sink_dev = nullptr, *sink_host = nullptr;
    bool sink_done = false;
    bool sink_pageable = false;  // pageable destination: parts go to the drain thread (hostio.cuh)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev = nullptr;
    HostStage *stage = nullptr;  // pageable host transfers (hostio.cuh), created on first use
    status_t sink_part(uint64_t first, uint64_t count) {
        if (count == 0) return PSACAK_OK;
        if (sink_pageable) return drain_part(*this, first, count);
        PSK_CUDA(cudaEventRecord(copy_ev, stream));
        PSK_CUDA(cudaStreamWaitEvent(copy_stream, copy_ev, 0));
        PSK_CUDA(cudaMemcpyAsync(sink_host + first, sink_dev + first, count * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, copy_stream));
        return PSACAK_OK;
    }

    // Workspace arena: one device buffer reused by every build.  Blocks are
    // carved from the top and released stack-wise (a block freed out of
    // order is reclaimed when everything above it is free).  A request that
    // does not fit goes to the stream-ordered pool instead, and the arena is
    // regrown to the observed high-water mark before the next build, so a
    // steady workload allocates nothing after its first build.
    struct Block {
        void *ptr;
        size_t size;
        bool in_arena;
        bool freed;
    };
    char *arena = nullptr;
    size_t arena_size = 0, arena_top = 0, arena_vtop = 0, arena_high = 0;
    std::vector<Block> blocks;

    // Called at the start of a public call, when no block is live: regrows
    // the arena to the high-water mark seen so far.
    status_t arena_prepare() {
        if (!blocks.empty()) return PSACAK_OK;
        arena_top = arena_vtop = 0;
        if (arena_high > arena_size) {
            PSK_CUDA(cudaStreamSynchronize(stream));
            if (arena) cudaFree(arena);
            arena = nullptr;
            arena_size = 0;
            // what the pool kept from the builds that outgrew the arena goes back
            PSK_CUDA(cudaMemPoolTrimTo(pool, 0));
            size_t want = arena_high + arena_high / 8 + (64u << 20);
            PSK_CUDA(cudaMalloc(&arena, want));
            arena_size = want;
        }
        return PSACAK_OK;
    }
    template <class T>
    status_t alloc(T **p, size_t count) {
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = 16;
        bytes = (bytes + 255) & ~(size_t)255;
        if (ws_cap && arena_vtop + bytes > ws_cap) {
            *p = nullptr;
            return set_error(PSACAK_ENOMEM, "device allocation of %zu bytes failed: workspace cap of %llu bytes",
                             bytes, (unsigned long long)ws_cap);
        }
        arena_vtop += bytes;
        if (arena_vtop > arena_high) arena_high = arena_vtop;
        if (arena && arena_top + bytes <= arena_size) {
            blocks.push_back(Block{arena + arena_top, bytes, true, false});
            *p = (T *)(arena + arena_top);
            arena_top += bytes;
            return PSACAK_OK;
        }
        void *q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, pool, stream);
        if (e != cudaSuccess) {
            arena_vtop -= bytes;
            *p = nullptr;
            return set_error(PSACAK_ENOMEM, "device allocation of %zu bytes failed: %s", bytes,
                             cudaGetErrorString(e));
        }
        blocks.push_back(Block{q, bytes, false, false});
        *p = (T *)q;
        return PSACAK_OK;
    }
    void release(void *p) {
        if (!p) return;
        for (size_t i = blocks.size(); i-- > 0;) {
            if (blocks[i].ptr == p && !blocks[i].freed) {
                blocks[i].freed = true;
                if (!blocks[i].in_arena) cudaFreeAsync(p, stream);
                break;
            }
        }
        while (!blocks.empty() && blocks.back().freed) {
            const Block &b = blocks.back();
            arena_vtop -= b.size;
            if (b.in_arena) arena_top = (size_t)((char *)b.ptr - arena);
            blocks.pop_back();
        }
    }
    // Copies `count` uint32 from device to host and waits for the stream.
    status_t read_u32(const uint32_t *d, uint32_t *h, size_t count = 1) {
        PSK_TRY(read_back(d, m_pinned, (uint32_t)count, stream));
        for (size_t i = 0; i < count; i++) h[i] = ((volatile uint32_t *)h_pinned)[i];
        return PSACAK_OK;
    }
    // Debug aid: when stage timing is on, waits for the stream and prints the
    // wall time since the previous mark.
    void mark(const char *what, uint32_t level) {
        if (!stage_timing) return;
        cudaStreamSynchronize(stream);
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        double t = ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
        if (stage_t0 > 0)
            fprintf(stderr, "[psacak] level %u %-24s %9.3f ms  workspace %.2f GB (peak %.2f GB)\n", level, what,
                    t - stage_t0, arena_vtop / 1e9, arena_high / 1e9);
        stage_t0 = t;
    }
    // Items per thread of the bucket scans' scatter and of the compactions
    // (schedule tile_items; 0 = 8).  Radix passes always use RADIX_IPT.
    int tile_ipt() const {
        uint32_t t = sched.tile_items;
        return (t == 12 || t == 16) ? (int)t : 8;
    }
    // Grows the onesweep status array to hold `tiles` tiles.
    status_t ensure_onesweep(uint64_t tiles) {
        if (tiles <= os.max_tiles) return PSACAK_OK;
        uint64_t want = tiles + tiles / 4 + 64;
        if (os.status) cudaFreeAsync(os.status, stream);
        os.status = nullptr;
        os.max_tiles = 0;
        PSK_CUDA(cudaMallocFromPoolAsync(&os.status, want * 256 * sizeof(uint64_t), pool, stream));
        // zeroed words read as "not ready" for every epoch
        PSK_CUDA(cudaMemsetAsync(os.status, 0, want * 256 * sizeof(uint64_t), stream));
        os.max_tiles = want;
        return PSACAK_OK;
    }
    // Grows the single-pass scan scratch to cover `n` items.
    status_t ensure_scan(uint64_t n) {
        const uint64_t tiles = ceil_div(n ? n : 1, LS_TILE_MIN) + 1;
        if (tiles <= ss.max_tiles) return PSACAK_OK;
        const uint64_t want = tiles + tiles / 4 + 64;
        if (ss.flags) cudaFreeAsync(ss.flags, stream);
        ss.flags = nullptr;
        ss.max_tiles = 0;
        PSK_CUDA(cudaMallocFromPoolAsync(&ss.flags, want * LS_MAX_FIELDS * sizeof(uint64_t), pool, stream));
        // zeroed words read as "not ready" for every epoch
        PSK_CUDA(cudaMemsetAsync(ss.flags, 0, want * LS_MAX_FIELDS * sizeof(uint64_t), stream));
        ss.max_tiles = want;
        return PSACAK_OK;
    }
    ScanEnv scan_env() { return ScanEnv{&ss, &os, d_err}; }
    // Single-pass scan (see lbscan.cuh) over n items.
    // `dn` (nullable): the item count is on the device, n is its bound.
    // `bytes`: algorithmic bytes of the launch for the profiler (0: no model).
    template <class T, class Op, class Load, class Store>
    status_t scan(Load ld, Store st, uint64_t n, T *total_out, Op op, const char *name, const uint32_t *dn = nullptr,
                  uint64_t bytes = 0) {
        PSK_TRY(ensure_scan(n));
        return lb_scan<T, Op>(ld, st, n, total_out, op, ss, os, d_err, stream, name, dn, bytes);
    }
    // Stable LSD radix sort of (key, value) pairs on bits [b0, b1); the
    // sorted data ends in (k1, v1) when *in1 is set, else in (k0, v0).
    // `hist_ready`: the digits were already counted into d_hist by the
    // keys' producer.
    template <class K, class V>
    status_t radix_sort(K *k0, V *v0, K *k1, V *v1, uint64_t n, int b0, int b1, int *in1, bool hist_ready = false,
                        const uint32_t *dn = nullptr) {
        PSK_TRY(ensure_onesweep(ceil_div(n, 8 * OS_BLOCK) + 1));
        return radix_sort_pairs<K, V>(k0, v0, k1, v1, n, b0, b1, d_hist, h_hist, m_hist, os, d_err, in1, stream, RADIX_IPT,
                                      hist_ready, dn);
    }
    // Single-pass stable compaction (see compact1).
    template <class Pred, class Emit>
    status_t compact(Pred pred, Emit emit, uint64_t n, uint32_t *count_out, const char *name) {
        PSK_TRY(ensure_onesweep(ceil_div(n, 8 * OS_BLOCK) + 1));
        return compact1(pred, emit, n, count_out, os, d_err, stream, name, tile_ipt());
    }
    status_t sync() {
        PSK_CUDA(cudaStreamSynchronize(stream));
        return PSACAK_OK;
    }
    // Fills in the trace's deferred hashes (one read-back for all levels).
    status_t resolve_trace() {
        if (pending_hash.empty()) return PSACAK_OK;
        uint32_t top = 0;
        for (auto &ph : pending_hash) top = ph.second + 1 > top ? ph.second + 1 : top;
        uint32_t h[2 * HASH_SLOTS];
        PSK_TRY(read_u32((const uint32_t *)d_hashes, h, 2 * top));
        for (auto &ph : pending_hash)
            trace[ph.first].hash = ((uint64_t)h[2 * ph.second + 1] << 32) | h[2 * ph.second];
        pending_hash.clear();
        return PSACAK_OK;
    }
    status_t check_device_error() {
        uint32_t e = 0;
        PSK_TRY(read_u32(d_err, &e));
        if (e) {
            PSK_CUDA(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), stream));
            if (e & DEVERR_TIMEOUT) return set_error(PSACAK_ETIMEOUT, "a bounded device wait ran out (0x%x)", e);
            return set_error(PSACAK_EINTERNAL, "device-side consistency check failed (0x%x)", e);
        }
        return PSACAK_OK;
    }
    // Ends a failed call: waits for the work already queued, then reports a
    // device-side timeout in preference to the host-side symptom it caused
    // (a count that did not add up), and clears the error word so that the
    // next call starts clean.  Cancellation and argument errors pass through.
    status_t fail(status_t st) {
        cudaStreamSynchronize(stream);
        if (st == PSACAK_ECANCELED || st == PSACAK_EINVAL) return st;
        uint32_t e = 0;
        if (read_u32(d_err, &e) != PSACAK_OK) return st;
        if (e) {
            cudaMemsetAsync(d_err, 0, sizeof(uint32_t), stream);
            cudaStreamSynchronize(stream);
            if (e & DEVERR_TIMEOUT) return set_error(PSACAK_ETIMEOUT, "a bounded device wait ran out (0x%x)", e);
        }
        return st;
    }
};

// RAII holder of a stream-ordered device allocation.
template <class T> struct DBuf {
    Ctx *ctx = nullptr;
    T *p = nullptr;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { reset(); }
    status_t init(Ctx &c, size_t count) {
        reset();
        ctx = &c;
        return c.alloc(&p, count);
    }
    void reset() {
        if (ctx && p) ctx->release(p);
        p = nullptr;
    }
    T *get() const { return p; }
    operator T *() const { return p; }
};

}  // namespace psk

struct psacak_ctx {
    psk::Ctx c;
};
