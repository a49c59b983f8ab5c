// induce_bucket.cu -- bucket-ordered induced scans of a byte level.
#include "ctx.cuh"
#include "induce.cuh"

namespace psk {

status_t induce_bucket8(Ctx &ctx, const uint8_t *text, uint64_t n, const uint32_t *types, const ByteGeom &hgeom,
                        const ByteGeom *dgeom, InduceMode mode, const uint32_t *sorted_lms, uint64_t n1,
                        uint32_t *sa, cudaStream_t s) {
    (void)ctx; (void)text; (void)n; (void)types; (void)hgeom; (void)dgeom; (void)mode; (void)sorted_lms;
    (void)n1; (void)sa; (void)s;
    return set_error(PSACAK_EINTERNAL, "bucket engine not built");
}

}  // namespace psk
