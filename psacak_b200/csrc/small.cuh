// small.cuh -- suffix arrays of short strings in shared memory (small.cu).
#pragma once

#include "common.cuh"

namespace psk {

struct Ctx;

// Longest string sorted in one CTA's shared memory.
constexpr uint32_t SMALL_MAX = 8192;

// The strings of one launch: either one string of length n at offset 0
// (offs == nullptr, count == 1), or the strings ids[0 .. count) of a packed
// batch, string i occupying [offs[i], offs[i+1]) (device arrays; ids best
// ordered longest first).  Each string's suffix array goes to the same
// offsets of the output.
struct SmallJobs {
    const uint64_t *offs;
    const uint32_t *ids;
    uint32_t count;
    uint64_t n;
    uint64_t symbols;  // symbols of all strings together (host-side accounting only)
};

// Suffix arrays of the strings of `jobs` (each of at most SMALL_MAX
// symbols, every symbol below sigma <= 65535), one CTA per string.
template <class C>
status_t small_sa(Ctx &ctx, const C *text, SmallJobs jobs, uint32_t sigma, uint32_t *sas, cudaStream_t s);

}  // namespace psk
