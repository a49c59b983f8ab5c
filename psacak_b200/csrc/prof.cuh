// prof.cuh -- optional per-kernel-class timing with CUDA events.
//
// When a context enables profiling, every instrumented launch records an
// event pair on its stream; after the build the pairs are resolved and
// accumulated per class (launches, device milliseconds, algorithmic bytes).
// With profiling off the hooks cost one thread-local pointer test.
#pragma once

#include <string.h>

#include <vector>

#include "common.cuh"

namespace psk {

struct ProfStat {
    const char *name;
    uint64_t launches = 0;
    uint64_t items = 0;
    uint64_t bytes = 0;
    double ms = 0.0;
};

struct Profiler {
    struct Pending {
        int cls;
        cudaEvent_t a, b;
        uint64_t items, bytes;
    };
    std::vector<ProfStat> stats;
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    int open_cls = -1;
    uint64_t open_items = 0, open_bytes = 0;
    cudaEvent_t open_a = nullptr;

    int cls_of(const char *name) {
        for (size_t i = 0; i < stats.size(); i++)
            if (strcmp(stats[i].name, name) == 0) return (int)i;
        ProfStat s;
        s.name = name;
        stats.push_back(s);
        return (int)stats.size() - 1;
    }
    cudaEvent_t get_event() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(const char *name, cudaStream_t s, uint64_t items, uint64_t bytes) {
        open_cls = cls_of(name);
        open_items = items;
        open_bytes = bytes;
        open_a = get_event();
        cudaEventRecord(open_a, s);
    }
    void end(cudaStream_t s) {
        if (open_cls < 0) return;
        cudaEvent_t b = get_event();
        cudaEventRecord(b, s);
        pending.push_back(Pending{open_cls, open_a, b, open_items, open_bytes});
        open_cls = -1;
    }
    // Call after the stream has been synchronised.
    void resolve() {
        for (auto &p : pending) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.a, p.b);
            ProfStat &st = stats[p.cls];
            st.launches++;
            st.ms += ms;
            st.items += p.items;
            st.bytes += p.bytes;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        resolve();
        stats.clear();
    }
    ~Profiler() {
        for (auto &p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

extern thread_local Profiler *t_prof;

// Wraps one kernel launch: PSK_PROF_LAUNCH(stream, "class", items, bytes, kernel<<<...>>>(...));
#define PSK_PROF_LAUNCH(stream, name, items, bytes, ...)                                        \
    do {                                                                                        \
        ::psk::Profiler *_p = ::psk::t_prof;                                                    \
        if (_p) _p->begin(name, stream, (uint64_t)(items), (uint64_t)(bytes));                   \
        __VA_ARGS__;                                                                            \
        if (_p) _p->end(stream);                                                                \
        PSK_KCOUNT();                                                                           \
    } while (0)

}  // namespace psk
