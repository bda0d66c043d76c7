// MLP warm start (placeholder until the tcgen05 GEMM lands).
#include "b2p_internal.cuh"

namespace b2p {
struct MlpState {};
void mlp_free(Ctx* ctx) { delete ctx->mlp; ctx->mlp = nullptr; }
}  // namespace b2p

using namespace b2p;
extern "C" {
int b2p_mlp_create(void* p, int, int, int, uint64_t) { static_cast<Ctx*>(p)->err = "mlp not built"; return B2P_EXECUTION_FAILED; }
int b2p_mlp_train_epoch(void* p, const float*, const float*, int, int, float, float*) { static_cast<Ctx*>(p)->err = "mlp not built"; return B2P_EXECUTION_FAILED; }
int b2p_mlp_infer(void* p, const float*, int, float*) { static_cast<Ctx*>(p)->err = "mlp not built"; return B2P_EXECUTION_FAILED; }
int b2p_gemm_bf16(void* p, int, int, int, const uint16_t*, int, const uint16_t*, int, float*) { static_cast<Ctx*>(p)->err = "mlp not built"; return B2P_EXECUTION_FAILED; }
}
