// hostio.cuh -- transfers between pageable host memory and the device.
//
// A copy from or to pageable memory goes through the CUDA driver's own
// staging, one thread and one buffer at a time (about a quarter of the PCIe
// rate on this hardware).  The builder stages those transfers itself: a
// ring of two pinned chunks per context, the host-side copies into or out of
// a chunk spread over a pool of host threads, and the DMA of one chunk
// overlapping the host copy of the next.  Pinned buffers need none of this
// and are copied directly.
#pragma once

#include <vector>

#include "common.cuh"

namespace psk {

struct Ctx;

// One host range and the device offset it corresponds to.
struct HostPiece {
    char *host;
    uint64_t dev_off;
    uint64_t bytes;
};

// True when `p` is pinned (page-locked and known to CUDA) host memory.
bool host_is_pinned(const void *p);

// d_dst[piece.dev_off ..] <- piece.host for every piece (device offsets
// ascending, non-overlapping), ordered on `s`; returns when the host ranges
// may be reused.
status_t staged_upload(Ctx &c, char *d_dst, const std::vector<HostPiece> &pieces, cudaStream_t s);

// piece.host <- d_src[piece.dev_off ..] for every piece, after the work
// already queued on `s`; returns when the host ranges hold the data.
status_t staged_download(Ctx &c, const char *d_src, const std::vector<HostPiece> &pieces, cudaStream_t s);

// Pageable destination of the final suffix array (see Ctx::sink_part): a
// host thread takes each finished part, moves it through the staging ring
// and copies it into `host` while the build goes on.  drain_begin starts the
// thread, drain_part (build thread, after the part's kernels are queued on
// the build stream) hands it a part, drain_end waits for every part and
// returns the first failure.
status_t drain_begin(Ctx &c, uint32_t *host, const uint32_t *dev);
status_t drain_part(Ctx &c, uint64_t first, uint64_t count);
status_t drain_end(Ctx &c);

// Releases the context's staging ring and host threads.
void host_stage_free(Ctx &c);

}  // namespace psk
