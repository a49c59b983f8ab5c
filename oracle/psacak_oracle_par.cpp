/*
 * psacak_oracle_par.cpp -- all-core CPU restatement of hucsmn/psacak's
 * pipelined induced sort for byte texts.  TEST AND BASELINE INFRASTRUCTURE
 * ONLY: the B200 builder never calls it; bench.py times it as the all-core
 * CPU baseline, and the tests check that it equals the serial restatement.
 *
 * The reference runs each induced scan of a byte text of >= 2 blocks
 * (src/psacak8.rs:11-15, :108-123) as a three-stage block pipeline
 * (src/pipeline.rs:33-111, :196-358; src/psacak8.rs:201-344, :410-498):
 *   fetch  (all threads): for the next block, the predecessor character c0,
 *          its successor c1 and the position j of every non-empty entry;
 *   induce (one thread):  the serial scan of the current block, using the
 *          fetched triple when it still matches the entry (else reading the
 *          text), writing targets inside the current or the next block
 *          directly and deferring the others;
 *   flush  (all threads): the deferred writes of the previous block.
 * Deferred targets lie at least two blocks ahead, and a block's flush is
 * waited for before the block after next is scanned, so every entry is in
 * place when its slot is scanned; a fetch that ran before a write simply
 * misses (the triple's j does not match) and the scan reads the text.
 * Shared slots are read and written with relaxed atomic accesses.
 *
 * The inner (u32) levels and the other steps run the serial restatement, as
 * in psacak_oracle.cpp.
 */
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace par {

static inline uint32_t ld(const uint32_t *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
static inline void st(uint32_t *p, uint32_t v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }

// A fixed set of worker threads running chunked jobs; the caller's thread
// keeps working while a job runs and waits for it later.  A job object is
// started once and must outlive the pool's use of it (a worker may still
// look at a finished job).
class Pool {
  public:
    struct Job {
        std::function<void(size_t, size_t)> fn;
        size_t n = 0, chunk = 1, nchunks = 0;
        std::atomic<size_t> next{0}, done{0};
        std::atomic<int> active{0};  // workers inside run_chunks of this job
    };
    explicit Pool(unsigned workers) {
        for (unsigned t = 0; t < workers; t++) threads_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : threads_) t.join();
    }
    // Starts fn over [0, n) in chunks; returns at once.
    void start(Job &job, size_t n, std::function<void(size_t, size_t)> fn) {
        job.fn = std::move(fn);
        job.n = n;
        size_t parts = threads_.empty() ? 1 : threads_.size() * 4;
        job.chunk = n / parts + 1;
        job.nchunks = n == 0 ? 0 : (n + job.chunk - 1) / job.chunk;
        job.next.store(0);
        job.done.store(0);
        if (threads_.empty()) {  // no workers: run it here
            run_chunks(job);
            return;
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            jobs_.push_back(&job);
        }
        cv_.notify_all();
    }
    // Waits for the job, taking chunks itself while any are left; on return
    // no worker refers to the job any more.
    void wait(Job &job) {
        run_chunks(job);
        while (job.done.load(std::memory_order_acquire) < job.nchunks) std::this_thread::yield();
        {
            std::lock_guard<std::mutex> g(mu_);
            for (size_t i = 0; i < jobs_.size(); i++)
                if (jobs_[i] == &job) {
                    jobs_.erase(jobs_.begin() + (long)i);
                    break;
                }
        }
        while (job.active.load(std::memory_order_acquire) > 0) std::this_thread::yield();
    }

  private:
    static void run_chunks(Job &job) {
        for (;;) {
            size_t c = job.next.fetch_add(1);
            if (c >= job.nchunks) return;
            size_t lo = c * job.chunk, hi = lo + job.chunk < job.n ? lo + job.chunk : job.n;
            job.fn(lo, hi);
            job.done.fetch_add(1, std::memory_order_release);
        }
    }
    void loop() {
        for (;;) {
            Job *job = nullptr;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [this] {
                    if (stop_) return true;
                    for (Job *j : jobs_)
                        if (j->next.load() < j->nchunks) return true;
                    return false;
                });
                if (stop_) return;
                for (Job *j : jobs_)
                    if (j->next.load() < j->nchunks) {
                        job = j;
                        job->active.fetch_add(1, std::memory_order_relaxed);
                        break;
                    }
            }
            if (job) {
                run_chunks(*job);
                job->active.fetch_sub(1, std::memory_order_release);
            }
        }
    }
    std::vector<std::thread> threads_;
    std::vector<Job *> jobs_;
    std::mutex mu_;
    std::condition_variable cv_;
    bool stop_ = false;
};

// Fetched (c0, c1, j) triples of one block; j = UINT32_MAX marks an empty slot.
struct RBuf {
    std::vector<uint8_t> c0, c1;
    std::vector<uint32_t> j;
    void fetch(Pool &pool, Pool::Job &job, const uint8_t *text, uint32_t *suf, size_t lo, size_t hi) {
        c0.resize(hi - lo);
        c1.resize(hi - lo);
        j.resize(hi - lo);
        pool.start(job, hi - lo, [this, text, suf, lo](size_t a, size_t b) {
            for (size_t i = a; i < b; i++) {
                uint32_t x = ld(suf + lo + i);
                if (x > 0) {
                    c0[i] = text[x - 1];
                    c1[i] = text[x];
                    j[i] = x - 1;
                } else {
                    j[i] = UINT32_MAX;
                }
            }
        });
    }
};

// Deferred (slot, value) writes of one block.
struct WBuf {
    std::vector<uint32_t> slot, val;
    void flush(Pool &pool, Pool::Job &job, uint32_t *suf) {
        pool.start(job, slot.size(), [this, suf](size_t a, size_t b) {
            for (size_t i = a; i < b; i++) st(suf + slot[i], val[i]);
        });
    }
    void clear() {
        slot.clear();
        val.clear();
    }
};

// One pipelined scan.  `backward` walks the blocks from the end; `scan` is
// called per block with the block's range, its read buffer and the write
// window [wlo, whi) (current and next block).
template <class Scan>
void pipeline(Pool &pool, const uint8_t *text, uint32_t *suf, size_t len, size_t bs, bool backward, Scan scan) {
    const size_t nblocks = (len + bs - 1) / bs;
    auto block = [&](size_t b, size_t &lo, size_t &hi) {
        if (!backward) {
            lo = b * bs;
            hi = lo + bs < len ? lo + bs : len;
        } else {
            hi = len - b * bs;
            lo = hi > bs ? hi - bs : 0;
        }
    };
    RBuf rb[2];
    WBuf wb[2];
    std::deque<Pool::Job> jobs;  // every job started by this scan, alive until it returns
    Pool::Job *fetch_job[2] = {nullptr, nullptr}, *flush_job[2] = {nullptr, nullptr};
    size_t lo, hi;
    block(0, lo, hi);
    fetch_job[0] = &jobs.emplace_back();
    rb[0].fetch(pool, *fetch_job[0], text, suf, lo, hi);
    for (size_t b = 0; b < nblocks; b++) {
        const int cur = (int)(b & 1), nxt = cur ^ 1;
        block(b, lo, hi);
        pool.wait(*fetch_job[cur]);
        size_t nlo = lo, nhi = hi;
        if (b + 1 < nblocks) {
            block(b + 1, nlo, nhi);
            fetch_job[nxt] = &jobs.emplace_back();
            rb[nxt].fetch(pool, *fetch_job[nxt], text, suf, nlo, nhi);
        }
        const size_t wlo = lo < nlo ? lo : nlo, whi = hi > nhi ? hi : nhi;
        wb[cur].clear();
        scan(lo, hi, rb[cur], wlo, whi, wb[cur]);
        if (flush_job[nxt]) {  // the previous block's deferred writes
            pool.wait(*flush_job[nxt]);
            flush_job[nxt] = nullptr;
        }
        flush_job[cur] = &jobs.emplace_back();
        wb[cur].flush(pool, *flush_job[cur], suf);
    }
    for (int k = 0; k < 2; k++)
        if (flush_job[k]) pool.wait(*flush_job[k]);
}

}  // namespace par

namespace oracle_par {

// Pipelined nonpar_induce_sort for bytes: the same scans as induce_sort8 in
// psacak_oracle.cpp (src/psacak8.rs:127-190), each block's triples prefetched
// and out-of-window writes deferred as in src/psacak8.rs:201-344.
void induce_sort8_par(const uint8_t *text, size_t len, uint32_t *suf, uint32_t *ptrs_head, uint32_t *ptrs_tail,
                      bool left_most, unsigned threads) {
    const size_t BS = 128 * 1024;  // src/psacak8.rs:12
    par::Pool pool(threads > 1 ? threads - 1 : 0);
    uint32_t ptrs[256];
    // L scan, from the sentinel suffix n - 1.
    memcpy(ptrs, ptrs_head, sizeof(ptrs));
    uint8_t prev_c0 = text[len - 1];
    size_t p = ptrs[prev_c0];
    par::st(suf + p, (uint32_t)(len - 1));
    p += 1;
    par::pipeline(pool, text, suf, len, BS, false,
                  [&](size_t lo, size_t hi, par::RBuf &rb, size_t wlo, size_t whi, par::WBuf &wb) {
                      for (size_t i = lo; i < hi; i++) {
                          uint32_t x = par::ld(suf + i);
                          if (x == 0) continue;
                          size_t j = x - 1;
                          uint8_t c0, c1;
                          if (rb.j[i - lo] == j) {
                              c0 = rb.c0[i - lo];
                              c1 = rb.c1[i - lo];
                          } else {
                              c0 = text[j];
                              c1 = text[j + 1];
                          }
                          if (c0 != prev_c0) {
                              ptrs[prev_c0] = (uint32_t)p;
                              p = ptrs[c0];
                              prev_c0 = c0;
                          }
                          if (c0 >= c1) {
                              if (p >= wlo && p < whi) par::st(suf + p, (uint32_t)j);
                              else {
                                  wb.slot.push_back((uint32_t)p);
                                  wb.val.push_back((uint32_t)j);
                              }
                              p += 1;
                              if (left_most) par::st(suf + i, 0);
                          }
                      }
                  });
    // S scan, backward from the tails.
    memcpy(ptrs, ptrs_tail, sizeof(ptrs));
    prev_c0 = 255;
    p = ptrs[prev_c0];
    par::pipeline(pool, text, suf, len, BS, true,
                  [&](size_t lo, size_t hi, par::RBuf &rb, size_t wlo, size_t whi, par::WBuf &wb) {
                      for (size_t i = hi; i-- > lo;) {
                          uint32_t x = par::ld(suf + i);
                          if (x == 0) continue;
                          size_t j = x - 1;
                          uint8_t c0, c1;
                          if (rb.j[i - lo] == j) {
                              c0 = rb.c0[i - lo];
                              c1 = rb.c1[i - lo];
                          } else {
                              c0 = text[j];
                              c1 = text[j + 1];
                          }
                          if (c0 != prev_c0) {
                              ptrs[prev_c0] = (uint32_t)p;
                              p = ptrs[c0];
                              prev_c0 = c0;
                          }
                          if (c0 <= c1 && p <= i) {
                              p -= 1;
                              if (p >= wlo && p < whi) par::st(suf + p, (uint32_t)j);
                              else {
                                  wb.slot.push_back((uint32_t)p);
                                  wb.val.push_back((uint32_t)j);
                              }
                              if (left_most) par::st(suf + i, 0);
                          }
                      }
                  });
}

}  // namespace oracle_par
