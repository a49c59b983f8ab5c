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
 * LMS-substring naming follows the reference's fastpar naming
 * (src/naming.rs:169-259): the sorted LMS substrings are split into one
 * chunk per thread, every chunk compares its substrings with their
 * predecessors and counts the new names, an exclusive sum of the counts
 * gives each chunk its first name, and the chunks write the names of their
 * substrings in parallel; bucket tails, compaction and translation stay
 * serial, as in the reference.
 *
 * The inner (u32) levels scan with the same block pipeline's fetch stage
 * (src/psacak32.rs:289-484, src/pipeline.rs:74-111): the (j, text[j],
 * text[j+1]) triples of the next 64Ki-slot block are read by all threads
 * while the serial scan works through the current one, using a fetched
 * triple when its j still matches the slot.  The in-workspace bucket
 * counters of the u32 levels shift entries as they grow, so the scan keeps
 * every write itself (the reference's flush stage, with its conflict and
 * shift handling, is not restated); the prefetch is what the pipeline buys
 * on a scan whose text reads miss the cache.
 */
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <utility>
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


// Fetched (j, text[j], text[j+1]) of the u32 level's slots [lo, hi).
struct RBuf32 {
    size_t lo = 0, hi = 0;
    std::vector<uint32_t> j, c0, c1;
    void fetch(par::Pool &pool, par::Pool::Job &job, const uint32_t *text, const uint32_t *suf, size_t len,
               size_t a, size_t b, uint32_t empty) {
        lo = a;
        hi = b;
        j.resize(b - a);
        c0.resize(b - a);
        c1.resize(b - a);
        pool.start(job, b - a, [this, text, suf, len, a, empty](size_t x0, size_t x1) {
            for (size_t i = x0; i < x1; i++) {
                uint32_t x = par::ld(suf + a + i);
                if (x > 0 && x < empty && x < len) {
                    j[i] = x - 1;
                    c0[i] = text[x - 1];
                    c1[i] = text[x];
                } else {
                    j[i] = UINT32_MAX;
                }
            }
        });
    }
    // the fetched characters of slot i holding predecessor j, if still valid
    bool get(size_t i, size_t jj, uint32_t &a, uint32_t &b) const {
        if (i < lo || i >= hi || j[i - lo] != jj) return false;
        a = c0[i - lo];
        b = c1[i - lo];
        return true;
    }
};

// Block pipeline of one u32 scan: fetch(block b + 1) runs while the scan is
// in block b.  `at(i)` is called whenever the scan reaches slot i and keeps
// the current and next blocks fetched.
struct Prefetch32 {
    par::Pool &pool;
    const uint32_t *text;
    const uint32_t *suf;
    size_t len, bs;
    bool backward;
    uint32_t empty;
    Prefetch32(par::Pool &p, const uint32_t *t, const uint32_t *s, size_t l, size_t b, bool back, uint32_t e)
        : pool(p), text(t), suf(s), len(l), bs(b), backward(back), empty(e) {}
    RBuf32 rb[2];
    std::deque<par::Pool::Job> jobs;
    par::Pool::Job *job[2] = {nullptr, nullptr};
    long cur = -1;  // block being scanned
    void range(long b, size_t &lo, size_t &hi) const {
        if (!backward) {
            lo = (size_t)b * bs;
            hi = lo + bs < len ? lo + bs : len;
        } else {
            hi = len - (size_t)b * bs;
            lo = hi > bs ? hi - bs : 0;
        }
    }
    long nblocks() const { return (long)((len + bs - 1) / bs); }
    void start(long b) {
        if (b >= nblocks()) return;
        size_t lo, hi;
        range(b, lo, hi);
        job[b & 1] = &jobs.emplace_back();
        rb[b & 1].fetch(pool, *job[b & 1], text, suf, len, lo, hi, empty);
    }
    void at(size_t i) {
        long b = backward ? (long)((len - 1 - i) / bs) : (long)(i / bs);
        if (b <= cur) return;
        while (cur < b) {
            cur++;
            if (cur == 0) start(0);
            if (job[cur & 1]) {
                pool.wait(*job[cur & 1]);
                job[cur & 1] = nullptr;
            }
            start(cur + 1);
        }
    }
    bool get(size_t i, size_t j, uint32_t &a, uint32_t &b) const {
        return rb[0].get(i, j, a, b) || rb[1].get(i, j, a, b);
    }
    ~Prefetch32() {
        for (int k = 0; k < 2; k++)
            if (job[k]) pool.wait(*job[k]);
    }
};

}  // namespace oracle_par

// The serial u32 scan of psacak_oracle.cpp (src/psacak32.rs:137-275) with
// the block prefetch above; identical writes, so identical results.
namespace oracle_par {

constexpr uint32_t EMPTY32 = 1u << 31;
static inline size_t decode_counter32(uint32_t x) { return (size_t)(0u - x); }
static inline uint32_t encode_counter32(size_t n) { return 0u - (uint32_t)n; }

void induce_sort32_par(const uint32_t *text, uint32_t *suf, size_t len, bool left_most, unsigned threads) {
    const size_t BS = 64 * 1024;  // src/psacak32.rs:15
    par::Pool pool(threads > 1 ? threads - 1 : 0);
    {
        size_t p = text[len - 1];
        if (p + 1 < len && suf[p + 1] == EMPTY32) {
            suf[p] = encode_counter32(1);
            suf[p + 1] = (uint32_t)(len - 1);
        } else {
            suf[p] = (uint32_t)(len - 1);
        }
    }
    {
        Prefetch32 pf(pool, text, suf, len, BS, false, EMPTY32);
        size_t i = 0;
        while (i < len) {
            pf.at(i);
            if (suf[i] > 0 && suf[i] < EMPTY32) {
                size_t j = suf[i] - 1;
                uint32_t c0, c1;
                if (!pf.get(i, j, c0, c1)) {
                    c0 = text[j];
                    c1 = text[j + 1];
                }
                size_t p = c0;
                if (c0 >= c1) {
                    if (suf[p] < EMPTY32) {
                        size_t n = 0;
                        while (n <= p && suf[p - n] <= EMPTY32) n++;
                        std::memmove(suf + p - n, suf + p + 1 - n, n * sizeof(uint32_t));
                        suf[p] = EMPTY32;
                        if (i > p - n) i -= 1;
                    }
                    if (suf[p] == EMPTY32) {
                        if (p + 1 < len && suf[p + 1] == EMPTY32) {
                            suf[p] = encode_counter32(1);
                            suf[p + 1] = (uint32_t)j;
                        } else {
                            suf[p] = (uint32_t)j;
                        }
                    } else {
                        size_t q = p + 1 + decode_counter32(suf[p]);
                        if (q < len && suf[q] == EMPTY32) {
                            suf[p] -= 1;
                            suf[q] = (uint32_t)j;
                        } else {
                            std::memmove(suf + p, suf + p + 1, (q - p - 1) * sizeof(uint32_t));
                            suf[q - 1] = (uint32_t)j;
                            if (i > p) i -= 1;
                        }
                    }
                    if (left_most) {
                        suf[i] = EMPTY32;
                    } else if (j + 2 < len) {
                        uint32_t c2 = text[j + 2];
                        if (!(c1 > c2 || (c1 == c2 && i > (size_t)c1))) suf[i] = EMPTY32;
                    }
                }
            }
            i += 1;
        }
    }
    for (size_t t = 0; t < len; t++) {
        if (suf[t] > EMPTY32) {
            size_t n = decode_counter32(suf[t]);
            std::memmove(suf + t, suf + t + 1, n * sizeof(uint32_t));
            suf[t + n] = EMPTY32;
        }
    }
    {
        Prefetch32 pf(pool, text, suf, len, BS, true, EMPTY32);
        size_t i = len - 1;
        for (;;) {
            pf.at(i);
            if (suf[i] > 0 && suf[i] < EMPTY32) {
                size_t j = suf[i] - 1;
                uint32_t c0, c1;
                if (!pf.get(i, j, c0, c1)) {
                    c0 = text[j];
                    c1 = text[j + 1];
                }
                size_t p = c0;
                if (c0 < c1 || (c0 == c1 && i < p)) {
                    if (suf[p] < EMPTY32) {
                        size_t n = 0;
                        while (p + n < len && suf[p + n] < EMPTY32) n++;
                        std::memmove(suf + p + 1, suf + p, n * sizeof(uint32_t));
                        suf[p] = EMPTY32;
                        if (i < p + n) i += 1;
                    }
                    if (suf[p] == EMPTY32) {
                        if (p > 0 && suf[p - 1] == EMPTY32) {
                            suf[p] = encode_counter32(1);
                            suf[p - 1] = (uint32_t)j;
                        } else {
                            suf[p] = (uint32_t)j;
                        }
                    } else {
                        size_t q = p - decode_counter32(suf[p]);
                        if (q > 0 && suf[q - 1] == EMPTY32) {
                            suf[p] -= 1;
                            suf[q - 1] = (uint32_t)j;
                        } else {
                            std::memmove(suf + q + 1, suf + q, (p - q) * sizeof(uint32_t));
                            suf[q] = (uint32_t)j;
                            if (i < p) i += 1;
                        }
                    }
                    if (left_most) suf[i] = EMPTY32;
                }
            }
            if (i == 0) break;
            i -= 1;
        }
    }
}

// fastpar naming's parallel part (src/naming.rs:169-236): per chunk of the
// sorted LMS substrings, the new-name flags (kept in the top bit of the
// entry) and their count; then each chunk writes the names of its
// substrings into work[pos / 2].  `differs(i0, i1)` compares two LMS
// substrings (the caller's fingerprint test).  Returns the name of the
// last substring + 1 (the name count k).
size_t name_chunks_par(uint32_t *lmssubs, size_t n, uint32_t *work, size_t wlen, unsigned threads,
                       const std::function<bool(size_t, size_t)> &differs) {
    par::Pool pool(threads > 1 ? threads - 1 : 0);
    const uint32_t HI = 1u << 31;
    const size_t parts = threads ? threads : 1;
    const size_t chunk = (n - 1 + parts - 1) / parts;
    const size_t nchunks = (n - 1 + chunk - 1) / chunk;
    std::vector<uint32_t> first(nchunks), k0(nchunks + 1, 0);
    for (size_t c = 0; c < nchunks; c++) first[c] = lmssubs[c * chunk];  // each chunk's predecessor
    {
        par::Pool::Job job;
        pool.start(job, nchunks, [&](size_t a, size_t b) {
            for (size_t c = a; c < b; c++) {
                size_t lo = 1 + c * chunk, hi = lo + chunk < n ? lo + chunk : n;
                size_t i0 = first[c];
                uint32_t cnt = 0;
                for (size_t i = lo; i < hi; i++) {
                    size_t i1 = lmssubs[i];
                    if (differs(i0, i1)) {
                        lmssubs[i] |= HI;
                        cnt++;
                    }
                    i0 = i1;
                }
                k0[c + 1] = cnt;
            }
        });
        pool.wait(job);
    }
    for (size_t c = 0; c < nchunks; c++) k0[c + 1] += k0[c];
    for (size_t i = 0; i < wlen; i++) work[i] = UINT32_MAX;
    work[lmssubs[0] / 2] = 0;
    {
        par::Pool::Job job;
        pool.start(job, nchunks, [&](size_t a, size_t b) {
            for (size_t c = a; c < b; c++) {
                size_t lo = 1 + c * chunk, hi = lo + chunk < n ? lo + chunk : n;
                uint32_t k = k0[c];
                for (size_t i = lo; i < hi; i++) {
                    uint32_t x = lmssubs[i];
                    if (x & HI) k++;
                    par::st(work + (x & ~HI) / 2, k);  // no slot is written twice
                }
            }
        });
        pool.wait(job);
    }
    return (size_t)k0[nchunks] + 1;
}

}  // namespace oracle_par
