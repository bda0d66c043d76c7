// Internal declarations shared by the libb2p translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/b2p.h"

namespace b2p {

// ---------------------------------------------------------------- errors
struct Error {
    int code;
    std::string msg;
};

int map_cuda_error(cudaError_t e);

#define B2P_CUDA(ctx, call)                                                                      \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(_e);                      \
            return ::b2p::map_cuda_error(_e);                                                    \
        }                                                                                        \
    } while (0)

#define B2P_LAUNCH(ctx)                                                                          \
    do {                                                                                         \
        cudaError_t _e = cudaGetLastError();                                                     \
        if (_e != cudaSuccess) {                                                                 \
            (ctx)->err = std::string("kernel launch: ") + cudaGetErrorString(_e);                \
            return ::b2p::map_cuda_error(_e);                                                    \
        }                                                                                        \
    } while (0)

// ---------------------------------------------------------------- device buffers
// Typed owning device allocation (cudaMallocAsync would tie lifetime to a stream;
// the engine keeps buffers across solves, so plain cudaMalloc).
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t count = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        count = 0;
    }
    // Grows (never shrinks) to at least n elements; contents are not preserved.
    cudaError_t reserve(size_t n) {
        if (n <= count && p) return cudaSuccess;
        release();
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e == cudaSuccess) count = n;
        return e;
    }
    size_t bytes() const { return count * sizeof(T); }
};

// ---------------------------------------------------------------- LP on the device
// Standard form, FP64, as uploaded, plus the stable transpose (CSR of A^T with
// row indices ascending inside each column -- the order in which the
// reference's scatter SpMV, src/sparse_matrix.cpp:175-185, accumulates).
struct DevLP {
    int m = 0, n = 0;
    int64_t nnz = 0;
    DBuf<int32_t> rowptr, colidx, t_rowptr, t_colidx;
    DBuf<double> vals, t_vals;
    DBuf<double> b, c, lb, ub;
    DBuf<uint8_t> is_eq;
    double bnorm = 0, cnorm = 0;  // FP64 2-norms of the original b and c
    double mean_row_len = 0, mean_col_len = 0;
    int max_row_len = 0, max_col_len = 0;
};

struct HalpernWork;   // halpern_engine.cu
struct BatchWork;     // batch_engine.cu
struct MlpState;      // mlp.cu

struct Ctx {
    int device = 0;
    int sm_count = 148;
    int l2_bytes = 0;
    cudaStream_t stream = nullptr;       // stream all work is issued on
    cudaStream_t own_stream = nullptr;   // the context's own stream
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    bool has_lp = false;
    int64_t lp_gen = 0;                  // bumped by every upload (engines key their derived copies on it)
    DevLP lp;
    // scratch for the GpuBackend primitives
    DBuf<int32_t> s_rowptr, s_colidx;
    DBuf<double> s_vals, s_x, s_y, s_z;
    DBuf<unsigned long long> s_red;
    DBuf<int32_t> s_flag;
    // CUB temp storage for setup-only sorts / scans
    DBuf<uint8_t> cub_tmp;
    HalpernWork* hw = nullptr;
    BatchWork* bw = nullptr;
    MlpState* mlp = nullptr;
    int64_t launches = 0;
};

// ---------------------------------------------------------------- helpers
inline unsigned grid_for(int64_t threads, int block, int sm_count, int per_sm = 16) {
    int64_t g = (threads + block - 1) / block;
    int64_t cap = (int64_t)sm_count * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

double now_ms();

// Builds the stable transpose of a CSR matrix on the device (setup only).
int build_transpose(Ctx* ctx, int m, int n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx,
                    const double* vals, int32_t* t_rowptr, int32_t* t_colidx, double* t_vals);

// Engine entry points (defined in their own translation units).
int ref_engine_solve(Ctx* ctx, const b2p_params* p, b2p_result* r, double* x_out, double* y_out);
int halpern_engine_solve(Ctx* ctx, const b2p_params* p, const double* x0, const double* y0, b2p_result* r,
                         double* x_out, double* y_out);
int halpern_kernel_timing(Ctx* ctx, const b2p_params* p, int reps, double* primal_ms, double* dual_ms,
                          double* primal_bytes, double* dual_bytes);
void halpern_free(Ctx* ctx);
void batch_free(Ctx* ctx);
void mlp_free(Ctx* ctx);

// Learned warm start (mlp.cu), used by the batch engine: training set from a batched
// solve's answers (device, external order), and warm starts predicted on the device.
int mlp_set_dataset(Ctx* ctx, const float* feat_host, int count, int n, int m, const double* x_dev,
                    const double* y_dev, const double* om_dev);
int mlp_predict_warm(Ctx* ctx, const float* feat_host, int count, int n, int m, double* x0, double* y0, double* om);

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Max over non-negative doubles through their bit patterns (monotone for +0..+inf).
// NaN is skipped, as std::max(acc, NaN) keeps acc.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
    if (!(v == v)) return;
    if (v <= 0.0) return;
    atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

}  // namespace b2p
