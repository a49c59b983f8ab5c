// gen.cu -- device-side i.i.d. texts for the serving simulation.
//
// Symbol i of a text is drawn from splitmix64(seed, i), so a text of any
// length is produced at memory speed without a host round trip.  Bytes are
// drawn from `alphabet` (up to 256 listed byte values); u32 symbols are
// uniform on [0, alphabet_size).
#include "ctx.cuh"
#include "../../include/psacak_b200_select.h"

namespace psk {
const char *last_error();
void clear_error();

__device__ __forceinline__ uint64_t sm64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct Alpha {
    uint8_t v[256];
};

__global__ void k_gen_u8(uint8_t *out, uint64_t n, Alpha a, uint32_t k, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = sm64(seed ^ (i * 0xd1b54a32d192ed03ull));
        out[i] = a.v[(uint32_t)(((r >> 32) * (uint64_t)k) >> 32)];
    }
}

__global__ void k_gen_u32(uint32_t *out, uint64_t n, uint32_t k, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = sm64(seed ^ (i * 0xd1b54a32d192ed03ull));
        out[i] = (uint32_t)(((r >> 32) * (uint64_t)k) >> 32);
    }
}
}  // namespace psk

using namespace psk;

extern "C" int psacak_gen_iid_dev(psacak_ctx *ctx, void *d_out, uint64_t n, int width, const uint8_t *alphabet,
                                  uint32_t alphabet_size, uint64_t seed, void *stream) {
    clear_error();
    if (!ctx || (n > 0 && !d_out) || alphabet_size == 0 || (width != 1 && width != 4))
        return set_error(PSACAK_EINVAL, "bad generator arguments");
    if (width == 1 && (!alphabet || alphabet_size > 256)) return set_error(PSACAK_EINVAL, "byte alphabet missing");
    Ctx &c = ctx->c;
    PSK_CUDA(cudaSetDevice(c.dev.id));
    cudaStream_t s = stream ? (cudaStream_t)stream : c.own_stream;
    if (n == 0) return PSACAK_OK;
    uint64_t g = ceil_div(n, 256);
    uint32_t grid = (uint32_t)(g < 16384 ? g : 16384);
    if (width == 1) {
        Alpha a;
        for (uint32_t i = 0; i < 256; i++) a.v[i] = i < alphabet_size ? alphabet[i] : 0;
        k_gen_u8<<<grid, 256, 0, s>>>((uint8_t *)d_out, n, a, alphabet_size, seed);
    } else {
        k_gen_u32<<<grid, 256, 0, s>>>((uint32_t *)d_out, n, alphabet_size, seed);
    }
    PSK_KCOUNT();
    PSK_LAUNCH_CHECK();
    return PSACAK_OK;
}
