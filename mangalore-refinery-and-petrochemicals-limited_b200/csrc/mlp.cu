// Learned warm start: a small MLP trained and run on the 5th-generation tensor cores.
//
// GEMM: C[M,N] (FP32) = A[M,K] . B[N,K]^T with A, B BF16 row-major (both
// K-major, "TN").  One CTA computes one 128 x 128 output tile:
//   * warp 0, one elected thread: TMA producer -- cp.async.bulk.tensor.2d loads of
//     128 x 64 BF16 tiles of A and B (128-byte swizzle) into a 3-stage shared
//     memory ring, completion signalled on per-stage mbarriers (expect_tx);
//   * warp 1, one elected thread: issues tcgen05.mma.cta_group::1.kind::f16
//     (M = 128, N = 128, K = 16 per instruction, BF16 x BF16 -> FP32) reading
//     both operands from shared memory through UMMA descriptors; the accumulator
//     lives in 128 TMEM columns; tcgen05.commit frees a stage when its MMAs finish;
//   * all 4 warps: tcgen05.ld (32 lanes x 16 columns per load) of their TMEM lane
//     quarter, then the FP32 store of the tile.
// No cluster, no multicast.  Every mbarrier wait is bounded: on timeout the
// kernel records an error code and leaves without touching the output.
// Transposed operands are materialised by small transpose kernels so the MMA
// path only ever sees the K-major layout.
//
// MLP: in -> hidden -> hidden -> out, GELU (tanh form), BF16 weights and
// activations, FP32 accumulation and FP32 master weights updated by Adam; the
// three GEMMs per layer of the backward pass (dX = dZ W, dW = dZ^T X) run on the
// same kernel with transposed copies written by the epilogue kernels.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include <algorithm>
#include <numeric>
#include <random>

#include "b2p_internal.cuh"

namespace b2p {

struct MlpState {
    int in = 0, hid = 0, out = 0, outp = 0;  // outp: out rounded up to a multiple of 8
    int maxb = 0;                           // batch capacity of the activation buffers
    long long step = 0;
    // FP32 master weights, Adam moments, gradients; BF16 weights and transposes
    DBuf<float> W1, b1, W2, b2, W3, b3;
    DBuf<float> m1, v1, m2, v2, m3, v3, mb1, vb1, mb2, vb2, mb3, vb3;
    DBuf<float> gW1, gb1, gW2, gb2, gW3, gb3;
    DBuf<__nv_bfloat16> W1h, W1t, W2h, W2t, W3h, W3t;
    // activations for one batch (rows = batch)
    DBuf<float> Xf, Tf, Z1, Z2, Y, G;  // G: FP32 GEMM scratch
    DBuf<__nv_bfloat16> Xh, Xt, H1, H1t, H2, H2t, dY, dYt, dZ, dZt;
    DBuf<double> loss;
    DBuf<int> err;
    // Adam on the device: hyper = {learning rate, 1 - beta1^t, 1 - beta2^t}, t in dstep
    DBuf<float> hyper;
    DBuf<long long> dstep;
    // split-K partial sums of the GEMMs whose output tiles alone would leave most SMs idle
    DBuf<float> ws;
    // one training epoch captured as a CUDA graph (for this data-set size and batch)
    cudaGraphExec_t epoch_exec = nullptr;
    int epoch_n = 0, epoch_batch = 0;
    long long epoch_launches = 0;  // kernels one replay launches
    ~MlpState() {
        if (epoch_exec) cudaGraphExecDestroy(epoch_exec);
    }
    // normalisation of inputs and targets: v_norm = (v - mean) / std
    DBuf<float> in_mean, in_std, out_mean, out_std;
    bool has_norm = false;
    // training set resident on the device (normalised, row-major) and the epoch order
    DBuf<float> DX, DT;
    DBuf<int32_t> perm;
    int dcount = 0;
};

void mlp_free(Ctx* ctx) {
    delete ctx->mlp;
    ctx->mlp = nullptr;
}

namespace {

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the completion of the phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
    const uint32_t addr = smem_u32(bar);
    for (long long spin = 0; spin < (1ll << 26); ++spin) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (spin > 64) __nanosleep(64);
    }
    atomicExch(err, code);
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor of a K-major tile with 128-byte swizzle: rows of
// 128 bytes, 8-row swizzle atoms 1024 bytes apart (SBO), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc_k_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;            // LBO (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;  // SBO
    d |= (uint64_t)1 << 46;            // version
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D FP32, A BF16, B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Three stages (about 100 KB of shared memory) let two CTAs share an SM -- and its TMEM, 128
// columns each -- so one CTA's epilogue overlaps the other's main loop and a 256 x 10,008
// output fits in one wave.
constexpr int GBM = 128, GBN = 128, GBK = 64, GSTAGES = 3;
constexpr int GTILE_A = GBM * GBK * 2, GTILE_B = GBN * GBK * 2;
constexpr size_t GEMM_SMEM = 1024 + GSTAGES * (GTILE_A + GTILE_B) + 256;

// C[M,N] = A[M,K] . B[N,K]^T ; A, B through tensor maps; C FP32 row-major, ldc elements.
// Split-K: CTA z of gridDim.z sums k-blocks [z kbs, (z + 1) kbs) into C + z split_stride.
__global__ void __launch_bounds__(128, 2)
k_gemm_tn_bf16(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, float* __restrict__ C,
               int M, int N, int K, int ldc, int kbs, size_t split_stride, int* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);  // SW128 tiles: 1024-aligned
    uint8_t* sA = base;
    uint8_t* sB = base + GSTAGES * GTILE_A;
    uint64_t* full = (uint64_t*)(sB + GSTAGES * GTILE_B);
    uint64_t* empty = full + GSTAGES;
    uint64_t* accum = empty + GSTAGES;
    uint32_t* tmem_slot = (uint32_t*)(accum + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
    const int kb0 = blockIdx.z * kbs;
    const int nkb = min((K + GBK - 1) / GBK - kb0, kbs);  // k-blocks of this split (>= 1 by construction)
    C += blockIdx.z * split_stride;

    if (warp == 0) {  // TMEM: 128 FP32 columns for the 128 x 128 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(GBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 32) {
        for (int s = 0; s < GSTAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    if (warp == 0 && lane == 0) {  // producer
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % GSTAGES;
            const uint32_t ph = (kb / GSTAGES) & 1;
            if (kb >= GSTAGES) ok = mbar_wait(&empty[s], ph ^ 1, err, 1);
            if (!ok) break;
            mbar_expect_tx(&full[s], GTILE_A + GTILE_B);
            tma_load_2d(sA + s * GTILE_A, &tmA, &full[s], (kb0 + kb) * GBK, m0);
            tma_load_2d(sB + s * GTILE_B, &tmB, &full[s], (kb0 + kb) * GBK, n0);
        }
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        const uint32_t idesc = idesc_bf16(GBM, GBN);
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % GSTAGES;
            const uint32_t ph = (kb / GSTAGES) & 1;
            ok = mbar_wait(&full[s], ph, err, 2);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t da = sdesc_k_sw128(smem_u32(sA + s * GTILE_A));
            const uint64_t db = sdesc_k_sw128(smem_u32(sB + s * GTILE_B));
#pragma unroll
            for (int k = 0; k < GBK / 16; ++k)  // 16 BF16 = 32 bytes per step inside the swizzle atom
                umma_bf16(tmem, da + 2 * k, db + 2 * k, idesc, (kb | k) != 0 ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(accum);
    }
    __syncwarp();
    // epilogue: warp w owns TMEM lanes (= tile rows) 32w .. 32w+31
    const bool acc_ok = mbar_wait(accum, 0, err, 3);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (acc_ok && ok) {
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c = 0; c < GBN / 16; ++c) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 16), v);
            if (row < M) {
                float* dst = C + (size_t)row * ldc + n0 + c * 16;
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (n0 + c * 16 + i < N) dst[i] = v[i];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GBN));
    }
}

// ---------------------------------------------------------------- tensor maps (host)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// rows x cols BF16 row-major (ld elements, ld % 8 == 0, 16-byte aligned base); box 64 x box_rows
bool make_map(CUtensorMap* map, const void* ptr, int rows, int cols, int ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn || ((uintptr_t)ptr & 15) || (ld % 8)) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C = sum of `splits` partial tiles (fixed order: deterministic)
__global__ void k_splitk_reduce(int M, int N, int ldc, int splits, size_t stride, const float* __restrict__ ws,
                                float* __restrict__ C) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)M * N;
         i += (long long)gridDim.x * blockDim.x) {
        const size_t o = (size_t)(i / N) * ldc + (size_t)(i % N);
        float acc = 0.0f;
        for (int z = 0; z < splits; ++z) acc += ws[z * stride + o];
        C[o] = acc;
    }
}

// C[M,N] = A[M,K] B[N,K]^T; all leading dimensions multiples of 8.  With a workspace, a GEMM
// whose output tiles would occupy fewer than half of the SMs and whose K spans at least
// 8 k-blocks is split along K (each split >= 4 k-blocks), the partial tiles summed by
// k_splitk_reduce.
int gemm_tn(Ctx* ctx, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C, int ldc, int M, int N,
            int K, int* err, DBuf<float>* ws = nullptr) {
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, M, K, lda, GBM) || !make_map(&tb, B, N, K, ldb, GBN)) {
        ctx->err = "gemm: tensor map rejected (alignment) or driver entry point missing";
        return B2P_INVALID_ARGUMENT;
    }
    static bool attr = false;
    if (!attr) {
        B2P_CUDA(ctx, cudaFuncSetAttribute(k_gemm_tn_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
        attr = true;
    }
    const int tiles = ((N + GBN - 1) / GBN) * ((M + GBM - 1) / GBM);
    const int nkb = (K + GBK - 1) / GBK;
    int splits = 1;
    if (ws && 2 * tiles <= ctx->sm_count && nkb >= 8) splits = std::max(1, std::min(nkb / 4, ctx->sm_count / tiles));
    const int kbs = (nkb + splits - 1) / splits;
    splits = (nkb + kbs - 1) / kbs;  // every split gets at least one k-block
    const size_t stride = (size_t)M * ldc;
    float* out = C;
    if (splits > 1) {
        B2P_CUDA(ctx, ws->reserve(stride * splits));
        out = ws->p;
    }
    dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM, splits);
    k_gemm_tn_bf16<<<grid, 128, GEMM_SMEM, ctx->stream>>>(ta, tb, out, M, N, K, ldc, kbs, stride, err);
    ctx->launches += 1;
    if (splits > 1) {
        k_splitk_reduce<<<grid_for((long long)M * N, 256, ctx->sm_count, 8), 256, 0, ctx->stream>>>(M, N, ldc, splits,
                                                                                                   stride, ws->p, C);
        ctx->launches += 1;
    }
    B2P_LAUNCH(ctx);
    return B2P_OK;
}

// ---------------------------------------------------------------- elementwise kernels
__device__ __forceinline__ float gelu(float x) {
    const float k = 0.7978845608028654f;  // sqrt(2/pi)
    return 0.5f * x * (1.0f + tanhf(k * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float k = 0.7978845608028654f;
    const float u = k * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k * (1.0f + 3.0f * 0.044715f * x * x);
}

// 32 x 32 tiles of a rows x cols matrix, one tile at a time per CTA of 32 x 8 threads:
// f(r, c) computes element (r, c) once (with its side effects); the BF16 result goes to
// out (row-major, ld_out; stores coalesced along c) and, through a shared-memory tile,
// to outT (its transpose, ld_t; stores coalesced along r).  Either output may be null.
constexpr int kTileThreadsY = 8;
template <typename F>
__device__ __forceinline__ void tile_pass(int rows, int cols, __nv_bfloat16* out, int ld_out, __nv_bfloat16* outT,
                                          int ld_t, F f) {
    __shared__ __nv_bfloat16 t[32][34];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tiles_c = (cols + 31) / 32, tiles = tiles_c * ((rows + 31) / 32);
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int r0 = (tile / tiles_c) * 32, c0 = (tile % tiles_c) * 32;
#pragma unroll
        for (int k = 0; k < 32; k += kTileThreadsY) {
            const int r = r0 + ty + k, c = c0 + tx;
            if (r < rows && c < cols) {
                const __nv_bfloat16 v = f(r, c);
                if (out) out[(size_t)r * ld_out + c] = v;
                t[ty + k][tx] = v;
            }
        }
        if (!outT) continue;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 32; k += kTileThreadsY) {
            const int c = c0 + ty + k, r = r0 + tx;
            if (r < rows && c < cols) outT[(size_t)c * ld_t + r] = t[tx][ty + k];
        }
        __syncthreads();
    }
}

// FP32 rows x cols (ld_in) -> BF16 copy (ld_out) and optional BF16 transpose (cols x rows, ld_t)
__global__ void k_to_bf16(int rows, int cols, const float* __restrict__ in, int ld_in, __nv_bfloat16* out, int ld_out,
                          __nv_bfloat16* outT, int ld_t) {
    tile_pass(rows, cols, out, ld_out, outT, ld_t,
              [&](int r, int c) { return __float2bfloat16(in[(size_t)r * ld_in + c]); });
}

// BF16 rows x cols -> BF16 transpose
__global__ void k_transpose_bf16(int rows, int cols, const __nv_bfloat16* __restrict__ in, int ld_in,
                                 __nv_bfloat16* __restrict__ out, int ld_out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)rows * cols;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        out[(size_t)c * ld_out + r] = in[(size_t)r * ld_in + c];
    }
}

// Z = G + bias (FP32 kept for the backward GELU'), H = GELU(Z) as BF16 and its transpose;
// rows >= valid are zeroed.
__global__ void k_bias_gelu(int rows, int valid, int cols, const float* __restrict__ G, const float* __restrict__ bias,
                            float* __restrict__ Z, __nv_bfloat16* __restrict__ H, __nv_bfloat16* __restrict__ Ht,
                            int ld_t) {
    tile_pass(rows, cols, H, cols, Ht, ld_t, [&](int r, int c) {
        const size_t i = (size_t)r * cols + c;
        const float z = r < valid ? G[i] + bias[c] : 0.0f;
        if (Z) Z[i] = z;
        return __float2bfloat16(r < valid ? gelu(z) : 0.0f);
    });
}

// Y = G + b3; squared error against T on the valid rows / real columns; dY = 2 (Y - T) / (valid * out)
__global__ void k_out_loss(int rows, int valid, int out, int outp, const float* __restrict__ G,
                           const float* __restrict__ bias, const float* __restrict__ T, float* __restrict__ Y,
                           __nv_bfloat16* __restrict__ dY, __nv_bfloat16* __restrict__ dYt, int ld_t, double* loss,
                           bool want_grad) {
    double part = 0.0;
    const float scale = 2.0f / ((float)valid * (float)out);
    tile_pass(rows, outp, want_grad ? dY : nullptr, outp, want_grad ? dYt : nullptr, ld_t, [&](int r, int c) {
        const size_t i = (size_t)r * outp + c;
        const float y = G[i] + bias[c];
        if (Y) Y[i] = y;
        float g = 0.0f;
        if (r < valid && c < out && T) {
            const float d = y - T[(size_t)r * out + c];
            part += (double)d * d;
            g = scale * d;
        }
        return __float2bfloat16(g);
    });
    if (loss) {
        part = warp_sum(part);
        if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(loss, part);
    }
}

// dZ = G * GELU'(Z) (BF16 + transpose), rows >= valid zeroed
__global__ void k_gelu_back(int rows, int valid, int cols, const float* __restrict__ G, const float* __restrict__ Z,
                            __nv_bfloat16* __restrict__ dZ, __nv_bfloat16* __restrict__ dZt, int ld_t) {
    tile_pass(rows, cols, dZ, cols, dZt, ld_t, [&](int r, int c) {
        const size_t i = (size_t)r * cols + c;
        return __float2bfloat16(r < valid ? G[i] * gelu_grad(Z[i]) : 0.0f);
    });
}

// db[c] = sum over rows of a BF16 gradient (FP32 accumulation); one thread per column
__global__ void k_colsum(int rows, int cols, const __nv_bfloat16* __restrict__ D, float* __restrict__ db) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int r = 0; r < rows; ++r) s += __bfloat162float(D[(size_t)r * cols + c]);
        db[c] = s;
    }
}

// One Adam update of element i; hyper = {learning rate, 1 - beta1^t, 1 - beta2^t}.
__device__ __forceinline__ float adam_update(size_t i, float* __restrict__ w, const float* __restrict__ g,
                                             float* __restrict__ m, float* __restrict__ v, const float* hyper) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - hyper[0] * (mi / hyper[1]) / (sqrtf(vi / hyper[2]) + 1e-8f);
    w[i] = wi;
    return wi;
}

// Adam of a bias vector (n elements).
__global__ void k_adam_vec(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, const float* __restrict__ hyper) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) adam_update(i, w, g, m, v, hyper);
}

// Adam on FP32 master weights (rows x cols, ld == cols) for the first live_rows rows, then
// their BF16 copy and its transpose (cols x rows, ld_t); hyper null: no update, copies only.
__global__ void k_adam(int rows, int cols, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, const float* __restrict__ hyper, __nv_bfloat16* __restrict__ wh,
                       __nv_bfloat16* __restrict__ wt, int ld_t, int live_rows) {
    tile_pass(rows, cols, wh, cols, wt, ld_t, [&](int r, int c) {
        const size_t i = (size_t)r * cols + c;
        const float wi = (hyper && r < live_rows) ? adam_update(i, w, g, m, v, hyper) : w[i];
        return __float2bfloat16(wi);
    });
}

// Start of an Adam step on the device: t += 1, the bias corrections of step t, and the
// learning rate when lr >= 0 (a negative lr keeps the rate already in hyper[0]).
__global__ void k_adam_begin(long long* __restrict__ step, float* __restrict__ hyper, float lr) {
    const long long t = ++*step;
    hyper[1] = 1.0f - powf(0.9f, (float)t);
    hyper[2] = 1.0f - powf(0.999f, (float)t);
    if (lr >= 0.0f) hyper[0] = lr;
}

// deterministic init: U(-a, a), a = 1/sqrt(fan_in) (the default of a linear layer)
__global__ void k_init_uniform(long long n, float a, unsigned long long seed, float* __restrict__ w, long long live) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ull + seed * 0xD1B54A32D192ED03ull + 1;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        w[i] = i < live ? (float)((2.0 * u - 1.0) * a) : 0.0f;
    }
}

// ---------------------------------------------------------------- learned warm start: data kernels
// Column mean and std of a row-major [rows x cols] block (two passes, FP64), std
// floored at floor_rel * (1 + |mean|).  `logit` takes log(max(v, 1e-30)) of every
// value first (primal weights).
template <typename T>
__global__ void k_col_stats(int rows, int cols, const T* __restrict__ src, long long ld, float floor_rel, bool logit,
                            float* __restrict__ mean, float* __restrict__ stdv) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int r = 0; r < rows; ++r) {
            double v = (double)src[(size_t)r * ld + c];
            s += logit ? log(fmax(v, 1e-30)) : v;
        }
        const double mu = s / rows;
        double q = 0.0;
        for (int r = 0; r < rows; ++r) {
            double v = (double)src[(size_t)r * ld + c];
            const double d = (logit ? log(fmax(v, 1e-30)) : v) - mu;
            q += d * d;
        }
        const double sd = sqrt(q / rows);
        mean[c] = (float)mu;
        stdv[c] = (float)fmax(sd, floor_rel * (1.0 + fabs(mu)));
    }
}

// Normalised training targets [rows x (n + m + 1)]: x (n), y (m), log(primal weight).
__global__ void k_build_targets(int rows, int n, int m, const double* __restrict__ x, const double* __restrict__ y,
                                const double* __restrict__ om, const float* __restrict__ mean,
                                const float* __restrict__ stdv, float* __restrict__ T) {
    const int out = n + m + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)rows * out;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / out), c = (int)(i % out);
        const double v = c < n ? x[(size_t)r * n + c]
                               : (c < n + m ? y[(size_t)r * m + (c - n)] : log(fmax(om[r], 1e-30)));
        T[i] = (float)((v - (double)mean[c]) / (double)stdv[c]);
    }
}

// rows x cols: dst = (src - mean) / std
__global__ void k_norm_rows(long long count, int cols, const float* __restrict__ src, const float* __restrict__ mean,
                            const float* __restrict__ stdv, float* __restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count * cols;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % cols);
        dst[i] = (src[i] - mean[c]) / stdv[c];
    }
}

// dst[r] = src[idx[r]] for r < valid, zero rows up to `rows` (rows x cols, row-major)
__global__ void k_gather_rows(int valid, int rows, int cols, const int32_t* __restrict__ idx,
                              const float* __restrict__ src, float* __restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)rows * cols;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i % cols);
        dst[i] = r < valid ? src[(size_t)idx[r] * cols + c] : 0.0f;
    }
}

// MLP output rows (ld outp) -> warm start of instances row0 .. row0+valid-1:
// x0 [n], y0 [m] (external order, FP64) and the primal weight exp(clamped log).
__global__ void k_denorm_warm(int valid, int outp, int n, int m, const float* __restrict__ Y,
                              const float* __restrict__ mean, const float* __restrict__ stdv, long long row0,
                              double* __restrict__ x0, double* __restrict__ y0, double* __restrict__ om) {
    const int out = n + m + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)valid * out;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / out), c = (int)(i % out);
        const double v = (double)Y[(size_t)r * outp + c] * (double)stdv[c] + (double)mean[c];
        const long long g = row0 + r;
        if (c < n) x0[g * n + c] = v;
        else if (c < n + m) y0[g * m + (c - n)] = v;
        else om[g] = exp(fmin(fmax(v, -30.0), 30.0));
    }
}

// ---------------------------------------------------------------- MLP host side
unsigned ew_grid(Ctx* ctx, long long n) { return grid_for(n, 256, ctx->sm_count, 8); }
// grid of a tile_pass kernel over a rows x cols matrix (blocks of 32 x 8 threads)
unsigned tile_grid(Ctx* ctx, long long rows, long long cols) {
    return grid_for(((rows + 31) / 32) * ((cols + 31) / 32) * 256, 256, ctx->sm_count, 8);
}
const dim3 kTileBlock(32, kTileThreadsY);

int check_err(Ctx* ctx, MlpState* s) {
    int e = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&e, s->err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    B2P_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (e) {
        ctx->err = "tensor-core GEMM: a bounded mbarrier wait timed out (code " + std::to_string(e) + ")";
        return B2P_TIMEOUT;
    }
    return B2P_OK;
}

int reserve_batch(Ctx* ctx, MlpState* s, int rows) {
    if (rows <= s->maxb) return B2P_OK;
    const int b = (rows + 7) & ~7;
    const int in = s->in, h = s->hid, op = s->outp;
    for (auto* d : {&s->Xf}) B2P_CUDA(ctx, d->reserve((size_t)b * in));
    B2P_CUDA(ctx, s->Tf.reserve((size_t)b * s->out));
    for (auto* d : {&s->Z1, &s->Z2}) B2P_CUDA(ctx, d->reserve((size_t)b * h));
    B2P_CUDA(ctx, s->Y.reserve((size_t)b * op));
    B2P_CUDA(ctx, s->G.reserve((size_t)std::max(b, h) * std::max(op, std::max(h, in))));
    for (auto* d : {&s->Xh, &s->Xt}) B2P_CUDA(ctx, d->reserve((size_t)b * in));
    for (auto* d : {&s->H1, &s->H1t, &s->H2, &s->H2t, &s->dZ, &s->dZt}) B2P_CUDA(ctx, d->reserve((size_t)b * h));
    for (auto* d : {&s->dY, &s->dYt}) B2P_CUDA(ctx, d->reserve((size_t)b * op));
    s->maxb = b;
    return B2P_OK;
}

// Forward for `rows` (multiple of 8) rows already in Xh/Xt; valid rows carry data.
int forward(Ctx* ctx, MlpState* s, int rows, int valid, bool keep) {
    const int in = s->in, h = s->hid, op = s->outp;
    cudaStream_t st = ctx->stream;
    int r;
    if ((r = gemm_tn(ctx, s->Xh.p, in, s->W1h.p, in, s->G.p, h, rows, h, in, s->err.p, &s->ws))) return r;
    k_bias_gelu<<<tile_grid(ctx, rows, h), kTileBlock, 0, st>>>(rows, valid, h, s->G.p, s->b1.p, s->Z1.p, s->H1.p,
                                                                    keep ? s->H1t.p : nullptr, rows);
    if ((r = gemm_tn(ctx, s->H1.p, h, s->W2h.p, h, s->G.p, h, rows, h, h, s->err.p, &s->ws))) return r;
    k_bias_gelu<<<tile_grid(ctx, rows, h), kTileBlock, 0, st>>>(rows, valid, h, s->G.p, s->b2.p, s->Z2.p, s->H2.p,
                                                                    keep ? s->H2t.p : nullptr, rows);
    if ((r = gemm_tn(ctx, s->H2.p, h, s->W3h.p, h, s->G.p, op, rows, op, h, s->err.p))) return r;
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    return B2P_OK;
}

// Loss and gradients of one batch (rows padded to 8; X, T already on the device in Xf/Tf)
int backward(Ctx* ctx, MlpState* s, int rows, int valid) {
    const int in = s->in, h = s->hid, op = s->outp, out = s->out;
    cudaStream_t st = ctx->stream;
    int r;
    k_out_loss<<<tile_grid(ctx, rows, op), kTileBlock, 0, st>>>(rows, valid, out, op, s->G.p, s->b3.p, s->Tf.p,
                                                                    s->Y.p, s->dY.p, s->dYt.p, rows, s->loss.p, true);
    k_colsum<<<ew_grid(ctx, op), 256, 0, st>>>(rows, op, s->dY.p, s->gb3.p);
    // dW3 = dY^T H2 : [op, h]
    if ((r = gemm_tn(ctx, s->dYt.p, rows, s->H2t.p, rows, s->gW3.p, h, op, h, rows, s->err.p))) return r;
    // dH2 = dY W3 : [rows, h]  (B = W3^T stored [h][op])
    if ((r = gemm_tn(ctx, s->dY.p, op, s->W3t.p, op, s->G.p, h, rows, h, op, s->err.p, &s->ws))) return r;
    k_gelu_back<<<tile_grid(ctx, rows, h), kTileBlock, 0, st>>>(rows, valid, h, s->G.p, s->Z2.p, s->dZ.p, s->dZt.p,
                                                                    rows);
    k_colsum<<<ew_grid(ctx, h), 256, 0, st>>>(rows, h, s->dZ.p, s->gb2.p);
    if ((r = gemm_tn(ctx, s->dZt.p, rows, s->H1t.p, rows, s->gW2.p, h, h, h, rows, s->err.p, &s->ws))) return r;
    if ((r = gemm_tn(ctx, s->dZ.p, h, s->W2t.p, h, s->G.p, h, rows, h, h, s->err.p, &s->ws))) return r;
    // dZ1 reuses the dZ buffers
    k_gelu_back<<<tile_grid(ctx, rows, h), kTileBlock, 0, st>>>(rows, valid, h, s->G.p, s->Z1.p, s->dZ.p, s->dZt.p,
                                                                    rows);
    k_colsum<<<ew_grid(ctx, h), 256, 0, st>>>(rows, h, s->dZ.p, s->gb1.p);
    if ((r = gemm_tn(ctx, s->dZt.p, rows, s->Xt.p, rows, s->gW1.p, in, h, in, rows, s->err.p, &s->ws))) return r;
    B2P_LAUNCH(ctx);
    ctx->launches += 6;
    return B2P_OK;
}

// One Adam step of all parameters; lr >= 0 sets the learning rate, a negative lr keeps the
// one in device memory (the captured training epoch sets it before each replay).
int adam_step(Ctx* ctx, MlpState* s, float lr) {
    s->step += 1;
    const int in = s->in, h = s->hid, op = s->outp;
    cudaStream_t st = ctx->stream;
    const float* hy = s->hyper.p;
    k_adam_begin<<<1, 1, 0, st>>>(s->dstep.p, s->hyper.p, lr);
    k_adam<<<tile_grid(ctx, h, in), kTileBlock, 0, st>>>(h, in, s->W1.p, s->gW1.p, s->m1.p, s->v1.p, hy, s->W1h.p,
                                                         s->W1t.p, h, h);
    k_adam<<<tile_grid(ctx, h, h), kTileBlock, 0, st>>>(h, h, s->W2.p, s->gW2.p, s->m2.p, s->v2.p, hy, s->W2h.p,
                                                        s->W2t.p, h, h);
    k_adam<<<tile_grid(ctx, op, h), kTileBlock, 0, st>>>(op, h, s->W3.p, s->gW3.p, s->m3.p, s->v3.p, hy, s->W3h.p,
                                                         s->W3t.p, op, s->out);
    k_adam_vec<<<ew_grid(ctx, h), 256, 0, st>>>(h, s->b1.p, s->gb1.p, s->mb1.p, s->vb1.p, hy);
    k_adam_vec<<<ew_grid(ctx, h), 256, 0, st>>>(h, s->b2.p, s->gb2.p, s->mb2.p, s->vb2.p, hy);
    k_adam_vec<<<ew_grid(ctx, s->out), 256, 0, st>>>(s->out, s->b3.p, s->gb3.p, s->mb3.p, s->vb3.p, hy);
    B2P_LAUNCH(ctx);
    ctx->launches += 7;
    return B2P_OK;
}

// stage `valid` rows of X (FP32 host, in cols) and T (out cols) into the padded device batch
int stage_batch(Ctx* ctx, MlpState* s, const float* X, const float* T, int valid, int rows) {
    const int in = s->in;
    cudaStream_t st = ctx->stream;
    B2P_CUDA(ctx, cudaMemsetAsync(s->Xf.p, 0, sizeof(float) * (size_t)rows * in, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(s->Xf.p, X, sizeof(float) * (size_t)valid * in, cudaMemcpyHostToDevice, st));
    if (T) B2P_CUDA(ctx, cudaMemcpyAsync(s->Tf.p, T, sizeof(float) * (size_t)valid * s->out, cudaMemcpyHostToDevice, st));
    k_to_bf16<<<tile_grid(ctx, rows, in), kTileBlock, 0, st>>>(rows, in, s->Xf.p, in, s->Xh.p, in, s->Xt.p, rows);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    return B2P_OK;
}

// refresh BF16 copies after a parameter upload (Adam with lr = 0 and no live rows)
int refresh_bf16(Ctx* ctx, MlpState* s) {
    const int in = s->in, h = s->hid, op = s->outp;
    cudaStream_t st = ctx->stream;
    k_adam<<<tile_grid(ctx, h, in), kTileBlock, 0, st>>>(h, in, s->W1.p, s->gW1.p, s->m1.p, s->v1.p, nullptr, s->W1h.p,
                                                         s->W1t.p, h, 0);
    k_adam<<<tile_grid(ctx, h, h), kTileBlock, 0, st>>>(h, h, s->W2.p, s->gW2.p, s->m2.p, s->v2.p, nullptr, s->W2h.p,
                                                        s->W2t.p, h, 0);
    k_adam<<<tile_grid(ctx, op, h), kTileBlock, 0, st>>>(op, h, s->W3.p, s->gW3.p, s->m3.p, s->v3.p, nullptr, s->W3h.p,
                                                         s->W3t.p, op, 0);
    B2P_LAUNCH(ctx);
    ctx->launches += 3;
    return B2P_OK;
}

// flat parameter layout: W1 [hid x in], b1 [hid], W2 [hid x hid], b2 [hid], W3 [out x hid], b3 [out]
struct Seg {
    float* dev;
    long long count;
};

std::vector<Seg> segments(MlpState* s, bool grads) {
    const long long in = s->in, h = s->hid, out = s->out;
    if (grads)
        return {{s->gW1.p, h * in}, {s->gb1.p, h}, {s->gW2.p, h * h}, {s->gb2.p, h}, {s->gW3.p, out * h}, {s->gb3.p, out}};
    return {{s->W1.p, h * in}, {s->b1.p, h}, {s->W2.p, h * h}, {s->b2.p, h}, {s->W3.p, out * h}, {s->b3.p, out}};
}

}  // namespace

// ---------------------------------------------------------------- learned warm start (called by the batch engine)
// Training set from the answers of the last batched solve, kept on the device:
// inputs = normalised parameter vectors, targets = normalised [x, y, log(primal
// weight)] of every instance (external order).  Sets the normalisation.
int mlp_set_dataset(Ctx* ctx, const float* feat_host, int count, int n, int m, const double* x_dev,
                    const double* y_dev, const double* om_dev) {
    MlpState* s = ctx->mlp;
    if (!s) {
        ctx->err = "no MLP: call b2p_mlp_create first";
        return B2P_INVALID_ARGUMENT;
    }
    if (s->out != n + m + 1) {
        ctx->err = "MLP output width must be n + m + 1 of the batch (" + std::to_string(n + m + 1) + ")";
        return B2P_INVALID_ARGUMENT;
    }
    const int in = s->in, out = s->out;
    cudaStream_t st = ctx->stream;
    for (auto* d : {&s->in_mean, &s->in_std}) B2P_CUDA(ctx, d->reserve(in));
    for (auto* d : {&s->out_mean, &s->out_std}) B2P_CUDA(ctx, d->reserve(out));
    B2P_CUDA(ctx, s->DX.reserve((size_t)count * in));
    B2P_CUDA(ctx, s->DT.reserve((size_t)count * out));
    DBuf<float> raw;
    B2P_CUDA(ctx, raw.reserve((size_t)count * in));
    B2P_CUDA(ctx, cudaMemcpyAsync(raw.p, feat_host, sizeof(float) * (size_t)count * in, cudaMemcpyHostToDevice, st));
    k_col_stats<float><<<ew_grid(ctx, in), 256, 0, st>>>(count, in, raw.p, in, 1e-6f, false, s->in_mean.p, s->in_std.p);
    k_col_stats<double><<<ew_grid(ctx, n), 256, 0, st>>>(count, n, x_dev, n, 1e-4f, false, s->out_mean.p, s->out_std.p);
    k_col_stats<double><<<ew_grid(ctx, m), 256, 0, st>>>(count, m, y_dev, m, 1e-4f, false, s->out_mean.p + n,
                                                          s->out_std.p + n);
    k_col_stats<double><<<1, 32, 0, st>>>(count, 1, om_dev, 1, 1e-4f, true, s->out_mean.p + n + m, s->out_std.p + n + m);
    // one scale per block (x, y): the root-mean-square of the block's column stds, so
    // that the squared error in normalised units is the relative L2 error of the
    // block -- the distance a warm start saves -- and near-constant columns weigh
    // no more than their share
    {
        std::vector<float> sd(out);
        B2P_CUDA(ctx, cudaMemcpyAsync(sd.data(), s->out_std.p, sizeof(float) * out, cudaMemcpyDeviceToHost, st));
        B2P_CUDA(ctx, cudaStreamSynchronize(st));
        for (int blk = 0; blk < 2; ++blk) {
            const int b0 = blk == 0 ? 0 : n, b1 = blk == 0 ? n : n + m;
            double q = 0.0;
            for (int c = b0; c < b1; ++c) q += (double)sd[c] * sd[c];
            const float rms = (float)std::max(std::sqrt(q / std::max(1, b1 - b0)), 1e-12);
            for (int c = b0; c < b1; ++c) sd[c] = rms;
        }
        B2P_CUDA(ctx, cudaMemcpyAsync(s->out_std.p, sd.data(), sizeof(float) * out, cudaMemcpyHostToDevice, st));
    }
    k_norm_rows<<<ew_grid(ctx, (long long)count * in), 256, 0, st>>>(count, in, raw.p, s->in_mean.p, s->in_std.p, s->DX.p);
    k_build_targets<<<ew_grid(ctx, (long long)count * out), 256, 0, st>>>(count, n, m, x_dev, y_dev, om_dev,
                                                                        s->out_mean.p, s->out_std.p, s->DT.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 6;
    B2P_CUDA(ctx, cudaStreamSynchronize(st));
    s->has_norm = true;
    s->dcount = count;
    return B2P_OK;
}

// Warm start of `count` instances of one shape from their parameter vectors:
// normalise, forward on the tensor cores, de-normalise into x0 [count x n],
// y0 [count x m] (external order) and primal weights (device, FP64).
int mlp_predict_warm(Ctx* ctx, const float* feat_host, int count, int n, int m, double* x0, double* y0, double* om) {
    MlpState* s = ctx->mlp;
    if (!s || !s->has_norm) {
        ctx->err = "no trained MLP with normalisation (b2p_mlp_dataset_from_batch or b2p_mlp_set_normalization)";
        return B2P_INVALID_ARGUMENT;
    }
    if (s->out != n + m + 1) {
        ctx->err = "MLP output width must be n + m + 1 of the batch (" + std::to_string(n + m + 1) + ")";
        return B2P_INVALID_ARGUMENT;
    }
    const int in = s->in;
    cudaStream_t st = ctx->stream;
    DBuf<float> raw;
    B2P_CUDA(ctx, raw.reserve((size_t)count * in));
    B2P_CUDA(ctx, cudaMemcpyAsync(raw.p, feat_host, sizeof(float) * (size_t)count * in, cudaMemcpyHostToDevice, st));
    const int chunk = 4096;
    int r = reserve_batch(ctx, s, std::min(count, chunk));
    if (r) return r;
    for (int off = 0; off < count; off += chunk) {
        const int valid = std::min(chunk, count - off);
        const int rows = (valid + 7) & ~7;
        B2P_CUDA(ctx, cudaMemsetAsync(s->Xf.p, 0, sizeof(float) * (size_t)rows * in, st));
        k_norm_rows<<<ew_grid(ctx, (long long)valid * in), 256, 0, st>>>(valid, in, raw.p + (size_t)off * in,
                                                                           s->in_mean.p, s->in_std.p, s->Xf.p);
        k_to_bf16<<<tile_grid(ctx, rows, in), kTileBlock, 0, st>>>(rows, in, s->Xf.p, in, s->Xh.p, in, s->Xt.p, rows);
        B2P_LAUNCH(ctx);
        ctx->launches += 2;
        if ((r = forward(ctx, s, rows, valid, false))) return r;
        k_out_loss<<<tile_grid(ctx, rows, s->outp), kTileBlock, 0, st>>>(
            rows, valid, s->out, s->outp, s->G.p, s->b3.p, nullptr, s->Y.p, nullptr, nullptr, 0, nullptr, false);
        k_denorm_warm<<<ew_grid(ctx, (long long)valid * s->out), 256, 0, st>>>(valid, s->outp, n, m, s->Y.p,
                                                                              s->out_mean.p, s->out_std.p, off, x0, y0,
                                                                              om);
        B2P_LAUNCH(ctx);
        ctx->launches += 2;
    }
    return check_err(ctx, s);
}

}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_mlp_create(void* p, int in_dim, int hidden, int out_dim, uint64_t seed) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (in_dim <= 0 || hidden <= 0 || out_dim <= 0 || in_dim % 8 || hidden % 8) {
        ctx->err = "b2p_mlp_create: in_dim and hidden must be positive multiples of 8";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    mlp_free(ctx);
    MlpState* s = new MlpState();
    ctx->mlp = s;
    s->in = in_dim;
    s->hid = hidden;
    s->out = out_dim;
    s->outp = (out_dim + 7) & ~7;
    const size_t in = in_dim, h = hidden, op = s->outp;
    for (auto* d : {&s->W1, &s->m1, &s->v1, &s->gW1}) B2P_CUDA(ctx, d->reserve(h * in));
    for (auto* d : {&s->W2, &s->m2, &s->v2, &s->gW2}) B2P_CUDA(ctx, d->reserve(h * h));
    for (auto* d : {&s->W3, &s->m3, &s->v3, &s->gW3}) B2P_CUDA(ctx, d->reserve(op * h));
    for (auto* d : {&s->b1, &s->mb1, &s->vb1, &s->gb1, &s->b2, &s->mb2, &s->vb2, &s->gb2}) B2P_CUDA(ctx, d->reserve(h));
    for (auto* d : {&s->b3, &s->mb3, &s->vb3, &s->gb3}) B2P_CUDA(ctx, d->reserve(op));
    for (auto* d : {&s->W1h, &s->W1t}) B2P_CUDA(ctx, d->reserve(h * in));
    for (auto* d : {&s->W2h, &s->W2t}) B2P_CUDA(ctx, d->reserve(h * h));
    for (auto* d : {&s->W3h, &s->W3t}) B2P_CUDA(ctx, d->reserve(op * h));
    B2P_CUDA(ctx, s->loss.reserve(1));
    B2P_CUDA(ctx, s->err.reserve(1));
    B2P_CUDA(ctx, s->hyper.reserve(4));
    B2P_CUDA(ctx, s->dstep.reserve(1));
    cudaStream_t st = ctx->stream;
    for (auto* d : {&s->m1, &s->v1, &s->gW1}) B2P_CUDA(ctx, cudaMemsetAsync(d->p, 0, d->bytes(), st));
    for (auto* d : {&s->m2, &s->v2, &s->gW2, &s->m3, &s->v3, &s->gW3}) B2P_CUDA(ctx, cudaMemsetAsync(d->p, 0, d->bytes(), st));
    for (auto* d : {&s->mb1, &s->vb1, &s->gb1, &s->mb2, &s->vb2, &s->gb2, &s->mb3, &s->vb3, &s->gb3})
        B2P_CUDA(ctx, cudaMemsetAsync(d->p, 0, d->bytes(), st));
    B2P_CUDA(ctx, cudaMemsetAsync(s->err.p, 0, sizeof(int), st));
    B2P_CUDA(ctx, cudaMemsetAsync(s->dstep.p, 0, sizeof(long long), st));
    B2P_CUDA(ctx, cudaMemsetAsync(s->hyper.p, 0, 4 * sizeof(float), st));
    k_init_uniform<<<ew_grid(ctx, h * in), 256, 0, st>>>(h * in, 1.0f / std::sqrt((float)in), seed * 6 + 1, s->W1.p, h * in);
    k_init_uniform<<<ew_grid(ctx, h), 256, 0, st>>>(h, 1.0f / std::sqrt((float)in), seed * 6 + 2, s->b1.p, h);
    k_init_uniform<<<ew_grid(ctx, h * h), 256, 0, st>>>(h * h, 1.0f / std::sqrt((float)h), seed * 6 + 3, s->W2.p, h * h);
    k_init_uniform<<<ew_grid(ctx, h), 256, 0, st>>>(h, 1.0f / std::sqrt((float)h), seed * 6 + 4, s->b2.p, h);
    k_init_uniform<<<ew_grid(ctx, op * h), 256, 0, st>>>(op * h, 1.0f / std::sqrt((float)h), seed * 6 + 5, s->W3.p,
                                                         (long long)out_dim * h);
    k_init_uniform<<<ew_grid(ctx, op), 256, 0, st>>>(op, 1.0f / std::sqrt((float)h), seed * 6 + 6, s->b3.p, out_dim);
    B2P_LAUNCH(ctx);
    ctx->launches += 6;
    int r = refresh_bf16(ctx, s);
    if (r) return r;
    B2P_CUDA(ctx, cudaStreamSynchronize(st));
    return B2P_OK;
}

int b2p_mlp_train_epoch(void* p, const float* X, const float* Y, int N, int batch, float lr, float* loss_out) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || !X || !Y || N <= 0 || batch <= 0) {
        ctx->err = "b2p_mlp_train_epoch: no MLP or empty data";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    const int b8 = (batch + 7) & ~7;
    int r = reserve_batch(ctx, s, b8);
    if (r) return r;
    B2P_CUDA(ctx, cudaMemsetAsync(s->loss.p, 0, sizeof(double), ctx->stream));
    for (int off = 0; off < N; off += batch) {
        const int valid = std::min(batch, N - off);
        const int rows = (valid + 7) & ~7;
        if ((r = stage_batch(ctx, s, X + (size_t)off * s->in, Y + (size_t)off * s->out, valid, rows))) return r;
        if ((r = forward(ctx, s, rows, valid, true))) return r;
        if ((r = backward(ctx, s, rows, valid))) return r;
        if ((r = adam_step(ctx, s, lr))) return r;
    }
    double loss = 0.0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&loss, s->loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if ((r = check_err(ctx, s))) return r;
    if (loss_out) *loss_out = (float)(loss / ((double)N * s->out));
    return B2P_OK;
}

int b2p_mlp_infer(void* p, const float* X, int N, float* Y_out) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || !X || !Y_out || N <= 0) {
        ctx->err = "b2p_mlp_infer: no MLP or empty input";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    const int chunk = 4096;
    int r = reserve_batch(ctx, s, std::min(N, chunk));
    if (r) return r;
    std::vector<float> tmp;
    for (int off = 0; off < N; off += chunk) {
        const int valid = std::min(chunk, N - off);
        const int rows = (valid + 7) & ~7;
        if ((r = stage_batch(ctx, s, X + (size_t)off * s->in, nullptr, valid, rows))) return r;
        if ((r = forward(ctx, s, rows, valid, false))) return r;
        k_out_loss<<<tile_grid(ctx, rows, s->outp), kTileBlock, 0, ctx->stream>>>(
            rows, valid, s->out, s->outp, s->G.p, s->b3.p, nullptr, s->Y.p, nullptr, nullptr, 0, nullptr, false);
        B2P_LAUNCH(ctx);
        ctx->launches += 1;
        B2P_CUDA(ctx, cudaMemcpy2DAsync(Y_out + (size_t)off * s->out, sizeof(float) * s->out, s->Y.p,
                                        sizeof(float) * s->outp, sizeof(float) * s->out, valid, cudaMemcpyDeviceToHost,
                                        ctx->stream));
    }
    return check_err(ctx, s);
}

int b2p_mlp_get_params(void* p, float* flat) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx || !ctx->mlp || !flat) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    size_t off = 0;
    for (const Seg& sg : segments(ctx->mlp, false)) {
        B2P_CUDA(ctx, cudaMemcpyAsync(flat + off, sg.dev, sizeof(float) * sg.count, cudaMemcpyDeviceToHost, ctx->stream));
        off += sg.count;
    }
    B2P_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return B2P_OK;
}

int b2p_mlp_set_params(void* p, const float* flat) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx || !ctx->mlp || !flat) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    size_t off = 0;
    for (const Seg& sg : segments(ctx->mlp, false)) {
        B2P_CUDA(ctx, cudaMemcpyAsync(sg.dev, flat + off, sizeof(float) * sg.count, cudaMemcpyHostToDevice, ctx->stream));
        off += sg.count;
    }
    int r = refresh_bf16(ctx, ctx->mlp);
    if (r) return r;
    B2P_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return B2P_OK;
}

int b2p_mlp_gradient(void* p, const float* X, const float* Y, int N, float* loss_out, float* grad_flat) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || !X || !Y || N <= 0) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    const int rows = (N + 7) & ~7;
    int r = reserve_batch(ctx, s, rows);
    if (r) return r;
    B2P_CUDA(ctx, cudaMemsetAsync(s->loss.p, 0, sizeof(double), ctx->stream));
    if ((r = stage_batch(ctx, s, X, Y, N, rows))) return r;
    if ((r = forward(ctx, s, rows, N, true))) return r;
    if ((r = backward(ctx, s, rows, N))) return r;
    double loss = 0.0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&loss, s->loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if ((r = check_err(ctx, s))) return r;
    if (loss_out) *loss_out = (float)(loss / ((double)N * s->out));
    if (grad_flat) {
        size_t off = 0;
        for (const Seg& sg : segments(s, true)) {
            B2P_CUDA(ctx, cudaMemcpyAsync(grad_flat + off, sg.dev, sizeof(float) * sg.count, cudaMemcpyDeviceToHost,
                                          ctx->stream));
            off += sg.count;
        }
        B2P_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return B2P_OK;
}

int b2p_mlp_train(void* p, int epochs, int batch, float lr_start, float lr_end, uint64_t seed, float* loss_out) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || s->dcount <= 0 || epochs <= 0 || batch <= 0) {
        ctx->err = "b2p_mlp_train: no MLP, no device training set, or empty schedule";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    const int N = s->dcount, in = s->in, out = s->out;
    const int b8 = (batch + 7) & ~7;
    int r = reserve_batch(ctx, s, b8);
    if (r) return r;
    B2P_CUDA(ctx, s->perm.reserve(N));
    cudaStream_t st = ctx->stream;
    std::vector<int32_t> order(N);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    // One epoch is a fixed sequence of launches -- the sample order lives in perm and the
    // learning rate in device memory -- so it is captured once as a CUDA graph and replayed
    // every epoch: no per-step host work (launches, tensor-map encoding) on the critical path.
    auto epoch_body = [&]() -> int {
        int q;
        for (int off = 0; off < N; off += batch) {
            const int valid = std::min(batch, N - off);
            const int rows = (valid + 7) & ~7;
            k_gather_rows<<<ew_grid(ctx, (long long)rows * in), 256, 0, st>>>(valid, rows, in, s->perm.p + off, s->DX.p,
                                                                              s->Xf.p);
            k_gather_rows<<<ew_grid(ctx, (long long)rows * out), 256, 0, st>>>(valid, rows, out, s->perm.p + off,
                                                                               s->DT.p, s->Tf.p);
            k_to_bf16<<<tile_grid(ctx, rows, in), kTileBlock, 0, st>>>(rows, in, s->Xf.p, in, s->Xh.p, in, s->Xt.p,
                                                                        rows);
            B2P_LAUNCH(ctx);
            ctx->launches += 3;
            if ((q = forward(ctx, s, rows, valid, true))) return q;
            if ((q = backward(ctx, s, rows, valid))) return q;
            if ((q = adam_step(ctx, s, -1.0f))) return q;
        }
        return B2P_OK;
    };
    const int steps_per_epoch = (N + batch - 1) / batch;
    if (!s->epoch_exec || s->epoch_n != N || s->epoch_batch != batch) {
        if (s->epoch_exec) {
            cudaGraphExecDestroy(s->epoch_exec);
            s->epoch_exec = nullptr;
        }
        // outside the capture: kernel attributes and the split-K workspace of every GEMM shape
        // (one forward / backward of a full batch; no parameter changes)
        const int rows0 = (std::min(batch, N) + 7) & ~7;
        if ((r = forward(ctx, s, rows0, std::min(batch, N), true))) return r;
        if ((r = backward(ctx, s, rows0, std::min(batch, N)))) return r;
        B2P_CUDA(ctx, cudaStreamSynchronize(st));
        const long long launches0 = ctx->launches, step0 = s->step;
        cudaGraph_t graph = nullptr;
        B2P_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int body = epoch_body();
        cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (body != B2P_OK) {
            if (graph) cudaGraphDestroy(graph);
            return body;
        }
        if (ce != cudaSuccess) {
            ctx->err = std::string("b2p_mlp_train: epoch capture: ") + cudaGetErrorString(ce);
            return B2P_EXECUTION_FAILED;
        }
        ce = cudaGraphInstantiate(&s->epoch_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) {
            s->epoch_exec = nullptr;
            ctx->err = std::string("b2p_mlp_train: epoch graph: ") + cudaGetErrorString(ce);
            return B2P_EXECUTION_FAILED;
        }
        s->epoch_launches = ctx->launches - launches0;
        ctx->launches = launches0;  // counted per replay below
        s->step = step0;
        s->epoch_n = N;
        s->epoch_batch = batch;
    }
    double loss = 0.0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        B2P_CUDA(ctx, cudaMemcpyAsync(s->perm.p, order.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
        const double cosw = 0.5 * (1.0 + std::cos(3.14159265358979323846 * ep / epochs));
        const float lr = (float)(lr_end + (lr_start - lr_end) * cosw);
        B2P_CUDA(ctx, cudaMemcpyAsync(s->hyper.p, &lr, sizeof(float), cudaMemcpyHostToDevice, st));
        B2P_CUDA(ctx, cudaMemsetAsync(s->loss.p, 0, sizeof(double), st));
        B2P_CUDA(ctx, cudaGraphLaunch(s->epoch_exec, st));
        ctx->launches += s->epoch_launches;
        s->step += steps_per_epoch;
        if (ep == epochs - 1) {
            B2P_CUDA(ctx, cudaMemcpyAsync(&loss, s->loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        if ((r = check_err(ctx, s))) return r;  // one sync per epoch: the order and lr buffers are reused
    }
    if (loss_out) *loss_out = (float)(loss / ((double)N * out));
    return B2P_OK;
}

int b2p_mlp_get_normalization(void* p, float* in_mean, float* in_std, float* out_mean, float* out_std) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || !s->has_norm || !in_mean || !in_std || !out_mean || !out_std) {
        ctx->err = "b2p_mlp_get_normalization: no normalisation set";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    B2P_CUDA(ctx, cudaMemcpyAsync(in_mean, s->in_mean.p, sizeof(float) * s->in, cudaMemcpyDeviceToHost, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(in_std, s->in_std.p, sizeof(float) * s->in, cudaMemcpyDeviceToHost, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(out_mean, s->out_mean.p, sizeof(float) * s->out, cudaMemcpyDeviceToHost, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(out_std, s->out_std.p, sizeof(float) * s->out, cudaMemcpyDeviceToHost, st));
    B2P_CUDA(ctx, cudaStreamSynchronize(st));
    return B2P_OK;
}

int b2p_mlp_set_normalization(void* p, const float* in_mean, const float* in_std, const float* out_mean,
                              const float* out_std) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    MlpState* s = ctx->mlp;
    if (!s || !in_mean || !in_std || !out_mean || !out_std) {
        ctx->err = "b2p_mlp_set_normalization: no MLP or null argument";
        return B2P_INVALID_ARGUMENT;
    }
    for (int i = 0; i < s->in; ++i)
        if (!(in_std[i] > 0.0f)) {
            ctx->err = "b2p_mlp_set_normalization: input std must be positive";
            return B2P_INVALID_ARGUMENT;
        }
    for (int i = 0; i < s->out; ++i)
        if (!(out_std[i] > 0.0f)) {
            ctx->err = "b2p_mlp_set_normalization: target std must be positive";
            return B2P_INVALID_ARGUMENT;
        }
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    for (auto* d : {&s->in_mean, &s->in_std}) B2P_CUDA(ctx, d->reserve(s->in));
    for (auto* d : {&s->out_mean, &s->out_std}) B2P_CUDA(ctx, d->reserve(s->out));
    B2P_CUDA(ctx, cudaMemcpyAsync(s->in_mean.p, in_mean, sizeof(float) * s->in, cudaMemcpyHostToDevice, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(s->in_std.p, in_std, sizeof(float) * s->in, cudaMemcpyHostToDevice, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(s->out_mean.p, out_mean, sizeof(float) * s->out, cudaMemcpyHostToDevice, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(s->out_std.p, out_std, sizeof(float) * s->out, cudaMemcpyHostToDevice, st));
    B2P_CUDA(ctx, cudaStreamSynchronize(st));
    s->has_norm = true;
    return B2P_OK;
}

int b2p_gemm_bf16(void* p, int M, int N, int K, const uint16_t* A, int trans_a, const uint16_t* B, int trans_b,
                  float* C) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const int Kp = (K + 7) & ~7, Np = (N + 7) & ~7;
    DBuf<__nv_bfloat16> a_in, b_in, a, b;
    DBuf<float> c;
    DBuf<int> err;
    B2P_CUDA(ctx, a_in.reserve((size_t)M * K));
    B2P_CUDA(ctx, b_in.reserve((size_t)N * K));
    B2P_CUDA(ctx, a.reserve((size_t)M * Kp));
    B2P_CUDA(ctx, b.reserve((size_t)N * Kp));
    B2P_CUDA(ctx, c.reserve((size_t)M * Np));
    B2P_CUDA(ctx, err.reserve(1));
    B2P_CUDA(ctx, cudaMemsetAsync(a.p, 0, a.bytes(), st));
    B2P_CUDA(ctx, cudaMemsetAsync(b.p, 0, b.bytes(), st));
    B2P_CUDA(ctx, cudaMemsetAsync(err.p, 0, sizeof(int), st));
    B2P_CUDA(ctx, cudaMemcpyAsync(a_in.p, A, sizeof(uint16_t) * (size_t)M * K, cudaMemcpyHostToDevice, st));
    B2P_CUDA(ctx, cudaMemcpyAsync(b_in.p, B, sizeof(uint16_t) * (size_t)N * K, cudaMemcpyHostToDevice, st));
    // A as M x K (K-major, ld Kp); given K x M when trans_a
    if (trans_a) k_transpose_bf16<<<ew_grid(ctx, (long long)M * K), 256, 0, st>>>(K, M, a_in.p, M, a.p, Kp);
    else B2P_CUDA(ctx, cudaMemcpy2DAsync(a.p, Kp * 2, a_in.p, K * 2, K * 2, M, cudaMemcpyDeviceToDevice, st));
    // B as N x K; given K x N unless trans_b
    if (!trans_b) k_transpose_bf16<<<ew_grid(ctx, (long long)N * K), 256, 0, st>>>(K, N, b_in.p, N, b.p, Kp);
    else B2P_CUDA(ctx, cudaMemcpy2DAsync(b.p, Kp * 2, b_in.p, K * 2, K * 2, N, cudaMemcpyDeviceToDevice, st));
    B2P_LAUNCH(ctx);
    int r = gemm_tn(ctx, a.p, Kp, b.p, Kp, c.p, Np, M, N, Kp, err.p);
    if (r) return r;
    B2P_CUDA(ctx, cudaMemcpy2DAsync(C, sizeof(float) * N, c.p, sizeof(float) * Np, sizeof(float) * N, M,
                                    cudaMemcpyDeviceToHost, st));
    int e = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2P_CUDA(ctx, cudaStreamSynchronize(st));
    if (e) {
        ctx->err = "tensor-core GEMM: a bounded mbarrier wait timed out (code " + std::to_string(e) + ")";
        return B2P_TIMEOUT;
    }
    return B2P_OK;
}

}  // extern "C"
