// Batched engine (placeholder until the persistent batch kernel lands).
#include "b2p_internal.cuh"

namespace b2p {
struct BatchWork {};
void batch_free(Ctx* ctx) { delete ctx->bw; ctx->bw = nullptr; }
}  // namespace b2p

using namespace b2p;
extern "C" {
int b2p_batch_upload(void* p, int, const int32_t*, const int32_t*, const int64_t*, const int32_t*, const int32_t*,
                     const double*, int, const int32_t*, const double*, const double*, const double*, const double*,
                     const uint8_t*) {
    static_cast<Ctx*>(p)->err = "batch engine not built";
    return B2P_EXECUTION_FAILED;
}
int b2p_batch_solve(void* p, const b2p_params*, const double*, const double*, const double*, int32_t*, int64_t*,
                    double*, double*, double*, b2p_result*) {
    static_cast<Ctx*>(p)->err = "batch engine not built";
    return B2P_EXECUTION_FAILED;
}
}
