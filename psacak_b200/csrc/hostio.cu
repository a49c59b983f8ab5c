// hostio.cu -- staged transfers of pageable host memory (see hostio.cuh).
#include "hostio.cuh"

#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <exception>
#include <mutex>
#include <new>
#include <thread>

#include "ctx.cuh"

namespace psk {

namespace {

constexpr uint64_t STAGE_CHUNK = 64ull << 20;  // bytes per ring slot
constexpr uint64_t COPY_TASK = 1ull << 20;     // bytes per host copy task
constexpr unsigned MAX_COPY_THREADS = 16;

struct CopyTask {
    char *dst;
    const char *src;
    uint64_t bytes;
};

// A fixed set of host threads that run one list of memcpy tasks at a time;
// the calling thread works on the list too.
class CopyPool {
  public:
    // Starts up to `workers` threads; if the system refuses one, the pool
    // works with those it has (the calling thread always takes part).
    explicit CopyPool(unsigned workers) {
        for (unsigned i = 0; i < workers; i++) {
            try {
                threads_.emplace_back([this] { loop(); });
            } catch (const std::exception &) {
                break;
            }
        }
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : threads_) t.join();
    }
    void run(const std::vector<CopyTask> &tasks) {
        if (tasks.empty()) return;
        if (threads_.empty() || tasks.size() == 1) {
            for (const CopyTask &t : tasks) memcpy(t.dst, t.src, t.bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &tasks;
            next_.store(0);
            pending_ = threads_.size();
            generation_++;
        }
        cv_.notify_all();
        work(tasks);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    void work(const std::vector<CopyTask> &tasks) {
        for (size_t i; (i = next_.fetch_add(1)) < tasks.size();) memcpy(tasks[i].dst, tasks[i].src, tasks[i].bytes);
    }
    void loop() {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
            if (stop_) return;
            seen = generation_;
            const std::vector<CopyTask> *job = job_;
            lk.unlock();
            work(*job);
            lk.lock();
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::vector<CopyTask> *job_ = nullptr;
    std::atomic<size_t> next_{0};
    size_t pending_ = 0;
    uint64_t generation_ = 0;
    bool stop_ = false;
};

}  // namespace

struct HostStage {
    char *ring = nullptr;  // two pinned slots of STAGE_CHUNK bytes
    cudaEvent_t ev[2] = {nullptr, nullptr};
    CopyPool *pool = nullptr;
    // drain session (pageable sink)
    struct Part {
        uint64_t first, count;
        cudaEvent_t ready;
    };
    std::thread drainer;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<Part> parts;           // handed over, not yet taken
    std::vector<cudaEvent_t> part_ev;  // one per part of a session, reused across sessions
    size_t nparts = 0;                 // parts of the current session
    bool closing = false;
    status_t status = PSACAK_OK;
    char err[256] = "";
    uint32_t *host = nullptr;
    const uint32_t *dev = nullptr;
};

bool host_is_pinned(const void *p) {
    cudaPointerAttributes pa{};
    const bool pinned = p && cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a query on pageable memory may leave an error behind
    return pinned;
}

static status_t stage_ready(Ctx &c) {
    if (!c.stage) c.stage = new (std::nothrow) HostStage();
    if (!c.stage) return set_error(PSACAK_ENOMEM, "staging: out of host memory");
    HostStage &st = *c.stage;
    if (!st.ring) PSK_CUDA(cudaHostAlloc((void **)&st.ring, 2 * STAGE_CHUNK, cudaHostAllocDefault));
    for (int i = 0; i < 2; i++)
        if (!st.ev[i]) PSK_CUDA(cudaEventCreateWithFlags(&st.ev[i], cudaEventDisableTiming));
    if (!st.pool) {
        unsigned hw = std::thread::hardware_concurrency();
        unsigned t = std::min(hw ? hw : 1u, MAX_COPY_THREADS);
        st.pool = new (std::nothrow) CopyPool(t - 1);
        if (!st.pool) return set_error(PSACAK_ENOMEM, "staging: out of host memory");
    }
    // the slots are free once the transfers of an earlier call have ended
    for (int i = 0; i < 2; i++) PSK_CUDA(cudaEventSynchronize(st.ev[i]));
    return PSACAK_OK;
}

// The byte range [pos, pos + len) of the pieces' concatenation as copy
// tasks between the pieces and buf; `to_buf` picks the direction.
static void chunk_tasks(const std::vector<HostPiece> &pieces, uint64_t pos, uint64_t len, char *buf, bool to_buf,
                        std::vector<CopyTask> &tasks) {
    tasks.clear();
    uint64_t start = 0;  // concatenation offset of the current piece
    for (const HostPiece &p : pieces) {
        const uint64_t a = std::max(pos, start), b = std::min(pos + len, start + p.bytes);
        for (uint64_t x = a; x < b; x += COPY_TASK) {
            const uint64_t k = std::min(COPY_TASK, b - x);
            char *h = p.host + (x - start);
            char *s = buf + (x - pos);
            tasks.push_back(to_buf ? CopyTask{s, h, k} : CopyTask{h, s, k});
        }
        start += p.bytes;
        if (start >= pos + len) break;
    }
}

static status_t check_pieces(const std::vector<HostPiece> &pieces, uint64_t *base, uint64_t *total) {
    *base = pieces.empty() ? 0 : pieces[0].dev_off;
    uint64_t t = 0;
    for (const HostPiece &p : pieces) {
        if (p.dev_off != *base + t) return set_error(PSACAK_EINTERNAL, "staged transfer: pieces are not contiguous");
        if (p.bytes && !p.host) return set_error(PSACAK_EINVAL, "staged transfer: null host range");
        t += p.bytes;
    }
    *total = t;
    return PSACAK_OK;
}

status_t staged_upload(Ctx &c, char *d_dst, const std::vector<HostPiece> &pieces, cudaStream_t s) {
    uint64_t base, total;
    PSK_TRY(check_pieces(pieces, &base, &total));
    if (total == 0) return PSACAK_OK;
    PSK_TRY(stage_ready(c));
    HostStage &st = *c.stage;
    std::vector<CopyTask> tasks;
    for (uint64_t k = 0, pos = 0; pos < total; k++) {
        const uint64_t len = std::min(STAGE_CHUNK, total - pos);
        const int slot = (int)(k & 1);
        char *buf = st.ring + slot * STAGE_CHUNK;
        PSK_CUDA(cudaEventSynchronize(st.ev[slot]));  // the DMA of chunk k - 2 has left this slot
        chunk_tasks(pieces, pos, len, buf, true, tasks);
        st.pool->run(tasks);
        PSK_CUDA(cudaMemcpyAsync(d_dst + base + pos, buf, len, cudaMemcpyHostToDevice, s));
        PSK_CUDA(cudaEventRecord(st.ev[slot], s));
        pos += len;
    }
    return PSACAK_OK;
}

status_t staged_download(Ctx &c, const char *d_src, const std::vector<HostPiece> &pieces, cudaStream_t s) {
    uint64_t base, total;
    PSK_TRY(check_pieces(pieces, &base, &total));
    if (total == 0) return PSACAK_OK;
    PSK_TRY(stage_ready(c));
    HostStage &st = *c.stage;
    const uint64_t nchunks = ceil_div(total, STAGE_CHUNK);
    auto enqueue = [&](uint64_t k) -> status_t {
        const uint64_t pos = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, total - pos);
        const int slot = (int)(k & 1);
        PSK_CUDA(cudaMemcpyAsync(st.ring + slot * STAGE_CHUNK, d_src + base + pos, len, cudaMemcpyDeviceToHost, s));
        PSK_CUDA(cudaEventRecord(st.ev[slot], s));
        return PSACAK_OK;
    };
    PSK_TRY(enqueue(0));
    std::vector<CopyTask> tasks;
    for (uint64_t k = 0; k < nchunks; k++) {
        // the DMA of chunk k + 1 (into the slot whose host copy finished in
        // the previous step) runs while the host empties chunk k
        if (k + 1 < nchunks) PSK_TRY(enqueue(k + 1));
        const int slot = (int)(k & 1);
        PSK_CUDA(cudaEventSynchronize(st.ev[slot]));
        const uint64_t pos = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, total - pos);
        chunk_tasks(pieces, pos, len, st.ring + slot * STAGE_CHUNK, false, tasks);
        st.pool->run(tasks);
    }
    return PSACAK_OK;
}

// The drain thread: every part waits for its event on the copy stream and
// goes through the two ring slots, the DMA of one slot overlapping the host
// copy of the other.
static void drain_loop(Ctx *cp) {
    Ctx &c = *cp;
    HostStage &st = *c.stage;
    cudaSetDevice(c.dev.id);
    auto fail = [&](cudaError_t e, const char *what) {
        std::lock_guard<std::mutex> g(st.mu);
        if (st.status == PSACAK_OK) {
            st.status = PSACAK_ECUDA;
            snprintf(st.err, sizeof(st.err), "output copy: %s failed: %s", what, cudaGetErrorString(e));
        }
    };
    std::vector<CopyTask> tasks;
    uint64_t k = 0;  // pieces issued, for the slot alternation
    for (;;) {
        HostStage::Part part;
        {
            std::unique_lock<std::mutex> lk(st.mu);
            st.cv.wait(lk, [&] { return st.closing || !st.parts.empty(); });
            if (st.parts.empty()) return;  // closing and nothing left
            part = st.parts.front();
            st.parts.erase(st.parts.begin());
        }
        cudaError_t e = cudaStreamWaitEvent(c.copy_stream, part.ready, 0);
        if (e != cudaSuccess) {
            fail(e, "cudaStreamWaitEvent");
            continue;
        }
        const uint64_t bytes = part.count * sizeof(uint32_t);
        const char *src = (const char *)(st.dev + part.first);
        char *dst = (char *)(st.host + part.first);
        // pieces of one part: piece j + 1 is issued before piece j is copied out
        int prev_slot = -1;
        uint64_t prev_off = 0, prev_len = 0;
        for (uint64_t off = 0;; off += STAGE_CHUNK) {
            const bool more = off < bytes;
            int slot = -1;
            uint64_t len = 0;
            if (more) {
                slot = (int)(k++ & 1);
                len = std::min(STAGE_CHUNK, bytes - off);
                e = cudaMemcpyAsync(st.ring + slot * STAGE_CHUNK, src + off, len, cudaMemcpyDeviceToHost,
                                    c.copy_stream);
                if (e == cudaSuccess) e = cudaEventRecord(st.ev[slot], c.copy_stream);
                if (e != cudaSuccess) {
                    fail(e, "cudaMemcpyAsync");
                    break;
                }
            }
            if (prev_slot >= 0) {
                e = cudaEventSynchronize(st.ev[prev_slot]);
                if (e != cudaSuccess) {
                    fail(e, "cudaEventSynchronize");
                    break;
                }
                tasks.clear();
                for (uint64_t x = 0; x < prev_len; x += COPY_TASK)
                    tasks.push_back(CopyTask{dst + prev_off + x, st.ring + prev_slot * STAGE_CHUNK + x,
                                             std::min(COPY_TASK, prev_len - x)});
                st.pool->run(tasks);
            }
            if (!more) break;
            prev_slot = slot;
            prev_off = off;
            prev_len = len;
        }
    }
}

status_t drain_begin(Ctx &c, uint32_t *host, const uint32_t *dev) {
    PSK_TRY(stage_ready(c));
    HostStage &st = *c.stage;
    st.host = host;
    st.dev = dev;
    st.parts.clear();
    st.nparts = 0;
    st.closing = false;
    st.status = PSACAK_OK;
    st.err[0] = 0;
    try {
        st.drainer = std::thread(drain_loop, &c);
    } catch (const std::exception &e) {
        return set_error(PSACAK_ENOMEM, "output copy thread: %s", e.what());
    }
    return PSACAK_OK;
}

status_t drain_part(Ctx &c, uint64_t first, uint64_t count) {
    if (count == 0) return PSACAK_OK;
    HostStage &st = *c.stage;
    if (st.nparts == st.part_ev.size()) {
        cudaEvent_t e;
        PSK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        st.part_ev.push_back(e);
    }
    cudaEvent_t ev = st.part_ev[st.nparts++];
    PSK_CUDA(cudaEventRecord(ev, c.stream));
    {
        std::lock_guard<std::mutex> g(st.mu);
        st.parts.push_back(HostStage::Part{first, count, ev});
    }
    st.cv.notify_one();
    return PSACAK_OK;
}

status_t drain_end(Ctx &c) {
    HostStage &st = *c.stage;
    {
        std::lock_guard<std::mutex> g(st.mu);
        st.closing = true;
    }
    st.cv.notify_one();
    if (st.drainer.joinable()) st.drainer.join();
    PSK_CUDA(cudaStreamSynchronize(c.copy_stream));
    if (st.status != PSACAK_OK) return set_error(st.status, "%s", st.err);
    return PSACAK_OK;
}

void host_stage_free(Ctx &c) {
    if (!c.stage) return;
    HostStage &st = *c.stage;
    if (st.drainer.joinable()) drain_end(c);
    for (cudaEvent_t e : st.part_ev) cudaEventDestroy(e);
    st.part_ev.clear();
    for (int i = 0; i < 2; i++)
        if (st.ev[i]) {
            cudaEventSynchronize(st.ev[i]);
            cudaEventDestroy(st.ev[i]);
        }
    if (st.ring) cudaFreeHost(st.ring);
    delete st.pool;
    delete c.stage;
    c.stage = nullptr;
}

}  // namespace psk
