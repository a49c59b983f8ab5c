// noalloc.cu -- suffix-array check that allocates no memory.
//
// Some callers cannot let a library allocate device memory while they run:
// a serving loop that checks suffix arrays between requests cannot afford
// cudaMalloc/cudaFree (they synchronise the whole device and stall every
// other stream), and a host application that owns the device's memory budget
// may forbid allocations by its plugins altogether.  For them this file
// offers psacak_check_sa8_noalloc: the same Burkhardt-Kaerkkaeinen check as
// psacak_check_sa8_dev, whose inverse-suffix-array scratch comes from a fixed
// array compiled into the library instead of the workspace.
//
// * The array holds PSACAK_NOALLOC_CHECK_MAX entries (8 MiB) plus a result
//   word.  Every GPU that loads the library keeps it until the process exits.
// * Host code cannot use the array's name as a device address: the address
//   is looked up with cudaGetSymbolAddress once per device, on the first call
//   made with that device current.
// * All calls share the array and leave their contents in it.  Each call
//   clears what must start cleared (the result word and the n entries it
//   uses) on the caller's stream; calls whose work overlaps on the GPU race.
// * No cudaMalloc, cudaFree or allocating library routine is called.
#include <mutex>

#include "ctx.cuh"
#include "level.cuh"

namespace psk {

const char *last_error();
void clear_error();

static __device__ __align__(256) uint32_t g_noalloc_check[PSACAK_NOALLOC_CHECK_MAX + 64];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
uint32_t *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.
status_t noalloc_scratch(uint32_t **out) {
    int dev = 0;
    PSK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(PSACAK_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        uint32_t *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_check);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_check)", __FILE__, __LINE__);
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return PSACAK_OK;
}
}  // namespace

}  // namespace psk

using namespace psk;

extern "C" int psacak_check_sa8_noalloc(const uint8_t *d_text, uint64_t n, const uint32_t *d_sa, int *ok,
                                        void *stream) {
    clear_error();
    if (!ok) return set_error(PSACAK_EINVAL, "null result pointer");
    if (n > 0 && (!d_text || !d_sa)) return set_error(PSACAK_EINVAL, "null text or suffix-array pointer");
    if (n > PSACAK_NOALLOC_CHECK_MAX)
        return set_error(PSACAK_EINVAL, "psacak_check_sa8_noalloc: n = %llu exceeds the fixed scratch of %u entries",
                         (unsigned long long)n, (unsigned)PSACAK_NOALLOC_CHECK_MAX);
    uint32_t *scratch = nullptr;
    PSK_TRY(noalloc_scratch(&scratch));
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *isa = scratch;
    uint32_t *bad = scratch + PSACAK_NOALLOC_CHECK_MAX;
    // check_sa clears *bad and the n isa entries before its kernels run.
    PSK_TRY(check_sa<uint8_t>(d_text, n, d_sa, isa, bad, s));
    uint32_t h_bad = 1;
    PSK_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    PSK_CUDA(cudaStreamSynchronize(s));
    *ok = h_bad == 0;
    return PSACAK_OK;
}
