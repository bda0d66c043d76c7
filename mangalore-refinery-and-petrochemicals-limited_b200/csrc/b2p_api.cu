// libb2p: device/context management, LP upload, and the GpuBackend primitives.
//
// Compiled with --fmad=false: the FP64 SpMV and vector primitives here round
// every multiply and add separately, as the reference host loops do
// (src/gpu_backend.cpp:60-69, 135-327), so results agree bit for bit with
// CSRMatrix::multiply (src/sparse_matrix.cpp:153-163).
#include <cub/cub.cuh>

#include <chrono>
#include <cmath>
#include <cstring>
#include <new>

#include "b2p_internal.cuh"

namespace b2p {

int map_cuda_error(cudaError_t e) {
    switch (e) {
        case cudaSuccess: return B2P_OK;
        case cudaErrorMemoryAllocation: return B2P_OUT_OF_MEMORY;
        case cudaErrorNoDevice:
        case cudaErrorInsufficientDriver:
        case cudaErrorInvalidDevice: return B2P_GPU_UNAVAILABLE;
        case cudaErrorInvalidValue: return B2P_INVALID_ARGUMENT;
        default: return B2P_EXECUTION_FAILED;
    }
}

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------- transpose (setup only)
__global__ void k_row_of(int m, const int32_t* __restrict__ rowptr, int32_t* __restrict__ row_of) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) row_of[k] = i;
}

__global__ void k_iota(int64_t nnz, int32_t* __restrict__ v) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        v[k] = (int32_t)k;
}

__global__ void k_count(int64_t nnz, const int32_t* __restrict__ colidx, int32_t* __restrict__ counts) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&counts[colidx[k]], 1);
}

__global__ void k_gather_t(int64_t nnz, const int32_t* __restrict__ perm, const int32_t* __restrict__ row_of,
                           const double* __restrict__ vals, int32_t* __restrict__ t_colidx,
                           double* __restrict__ t_vals) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
        int32_t k = perm[p];
        t_colidx[p] = row_of[k];
        t_vals[p] = vals[k];
    }
}

int build_transpose(Ctx* ctx, int m, int n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx,
                    const double* vals, int32_t* t_rowptr, int32_t* t_colidx, double* t_vals) {
    cudaStream_t s = ctx->stream;
    B2P_CUDA(ctx, cudaMemsetAsync(t_rowptr, 0, sizeof(int32_t) * (n + 1), s));
    if (nnz == 0) return B2P_OK;
    DBuf<int32_t> row_of, keys_out, perm_in, perm_out;
    B2P_CUDA(ctx, row_of.reserve(nnz));
    B2P_CUDA(ctx, keys_out.reserve(nnz));
    B2P_CUDA(ctx, perm_in.reserve(nnz));
    B2P_CUDA(ctx, perm_out.reserve(nnz));
    unsigned g = grid_for(std::max<int64_t>(m, 1), 256, ctx->sm_count);
    k_row_of<<<g, 256, 0, s>>>(m, rowptr, row_of.p);
    unsigned gz = grid_for(nnz, 256, ctx->sm_count);
    k_iota<<<gz, 256, 0, s>>>(nnz, perm_in.p);
    k_count<<<gz, 256, 0, s>>>(nnz, colidx, t_rowptr + 1);
    B2P_LAUNCH(ctx);
    int end_bit = 1;
    while (end_bit < 31 && (1LL << end_bit) <= n) ++end_bit;
    // Stable LSD radix sort by column: entries of one column keep their row-major
    // order, so row indices ascend inside every column of the transpose.
    size_t tmp_sort = 0, tmp_scan = 0;
    B2P_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, colidx, keys_out.p, perm_in.p, perm_out.p,
                                                  (int)nnz, 0, end_bit, s));
    B2P_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, tmp_scan, t_rowptr + 1, t_rowptr + 1, n, s));
    B2P_CUDA(ctx, ctx->cub_tmp.reserve(std::max(tmp_sort, tmp_scan)));
    size_t tb = ctx->cub_tmp.bytes();
    B2P_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->cub_tmp.p, tb, colidx, keys_out.p, perm_in.p, perm_out.p,
                                                  (int)nnz, 0, end_bit, s));
    tb = ctx->cub_tmp.bytes();
    B2P_CUDA(ctx, cub::DeviceScan::InclusiveSum(ctx->cub_tmp.p, tb, t_rowptr + 1, t_rowptr + 1, n, s));
    k_gather_t<<<gz, 256, 0, s>>>(nnz, perm_out.p, row_of.p, vals, t_colidx, t_vals);
    B2P_LAUNCH(ctx);
    ctx->launches += 4;
    // temporaries are freed on return; make sure the stream is done with them
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    return B2P_OK;
}

// ---------------------------------------------------------------- validation
// CSRMatrix::is_valid (src/sparse_matrix.cpp:187-207): indices in range and strictly ascending.
__global__ void k_validate_csr(int m, int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                               int32_t* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int prev = -1;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int c = colidx[k];
            if (c < 0 || c >= n || c <= prev) { atomicExch(bad, i + 1); break; }
            prev = c;
        }
    }
}

static int host_rowptr_ok(int m, int64_t nnz, const int32_t* rowptr) {
    if (rowptr[0] != 0 || (int64_t)rowptr[m] != nnz) return 0;
    for (int i = 0; i < m; ++i)
        if (rowptr[i + 1] < rowptr[i]) return 0;
    return 1;
}

// ---------------------------------------------------------------- GpuBackend primitives
__global__ void k_spmv_f64(int m, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                           const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) sum += vals[k] * x[colidx[k]];
        y[i] = sum;
    }
}

__global__ void k_vec(int op, size_t n, double alpha, const double* __restrict__ a, const double* __restrict__ b,
                      double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double r;
        switch (op) {
            case B2P_VEC_ADD: r = a[i] + b[i]; break;
            case B2P_VEC_SUB: r = a[i] - b[i]; break;
            case B2P_VEC_SCALE: r = alpha * a[i]; break;
            default: r = alpha * a[i] + b[i]; break;
        }
        out[i] = r;
    }
}

// Deterministic two-pass FP64 reduction: fixed-size grid, per-block partials in a
// fixed order, then one block sums the partials in index order.
constexpr int kRedBlocks = 256;
constexpr int kRedThreads = 256;

__global__ void k_dot_partial(size_t n, const double* __restrict__ a, const double* __restrict__ b,
                              double* __restrict__ partial) {
    __shared__ double sh[kRedThreads / 32];
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += a[i] * (b ? b[i] : a[i]);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) t += sh[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_sum_partials(int count, const double* __restrict__ partial, double* __restrict__ out) {
    __shared__ double sh[kRedThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) s += partial[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) t += sh[w];
        out[0] = t;
    }
}

struct PhaseTimer {
    cudaEvent_t e[4];
    bool ok = false;
    PhaseTimer() {
        ok = true;
        for (auto& x : e)
            if (cudaEventCreate(&x) != cudaSuccess) ok = false;
    }
    ~PhaseTimer() {
        for (auto& x : e) cudaEventDestroy(x);
    }
    void fill(b2p_timing_t* t, double host_t0) {
        if (!t || !ok) return;
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, e[0], e[1]);
        cudaEventElapsedTime(&b, e[1], e[2]);
        cudaEventElapsedTime(&c, e[2], e[3]);
        t->h2d_time_ms = a;
        t->kernel_time_ms = b;
        t->d2h_time_ms = c;
        double total = now_ms() - host_t0;
        t->sync_time_ms = std::max(0.0, total - (a + b + c));
        t->total_gpu_time_ms = total;
    }
};

}  // namespace b2p

using namespace b2p;

static Ctx* as_ctx(void* p) { return static_cast<Ctx*>(p); }

extern "C" {

void b2p_params_default(b2p_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->engine = B2P_ENGINE_REFERENCE;
    p->precision = B2P_FP64;
    p->max_iterations = 50000;
    p->feasibility_tolerance = 1e-7;
    p->primal_step_size = 0.01;
    p->dual_step_size = 0.01;
    p->adaptive_step_size = 1;
    p->check_frequency = 100;
    p->eps_rel_kkt = 1e-6;
    p->check_every = 64;
    p->ruiz_iterations = 10;
    p->reflection = 1.0;
    p->restart_sufficient = 0.2;
    p->restart_necessary = 0.8;
    p->restart_artificial = 0.36;
    p->primal_weight = 0.0;
    p->step_safety = 0.998;
    p->refinement_rounds = -1;
    p->time_limit_s = 0.0;
    p->lanes_per_row = 0;
    p->eps_objective = 0.0;
    p->eps_infeasible = 1e-8;
}

int b2p_device_info(int device, b2p_device_info_t* out) {
    if (!out) return B2P_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= device || device < 0) {
        std::snprintf(out->device_name, sizeof(out->device_name), "None");
        std::snprintf(out->status_message, sizeof(out->status_message), "no CUDA device %d: %s", device,
                      e != cudaSuccess ? cudaGetErrorString(e) : "index out of range");
        return B2P_GPU_UNAVAILABLE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return B2P_GPU_UNAVAILABLE;
    std::snprintf(out->device_name, sizeof(out->device_name), "%s", prop.name);
    out->total_memory_bytes = prop.totalGlobalMem;
    out->compute_capability_major = prop.major;
    out->compute_capability_minor = prop.minor;
    out->multiprocessor_count = prop.multiProcessorCount;
    out->l2_cache_bytes = prop.l2CacheSize;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) out->free_memory_bytes = fr;
    cudaSetDevice(cur);
    // The kernels are built for sm_100a only.
    out->is_available = (prop.major == 10 && prop.minor == 0) ? 1 : 0;
    std::snprintf(out->status_message, sizeof(out->status_message), "%s (sm_%d%d, %d SMs, %.1f GiB)%s", prop.name,
                  prop.major, prop.minor, prop.multiProcessorCount, prop.totalGlobalMem / 1073741824.0,
                  out->is_available ? "" : ": this library is built for sm_100a only");
    return out->is_available ? B2P_OK : B2P_GPU_UNAVAILABLE;
}

int b2p_ctx_create(int device, void** ctx_out) {
    if (!ctx_out) return B2P_INVALID_ARGUMENT;
    *ctx_out = nullptr;
    b2p_device_info_t info;
    int st = b2p_device_info(device, &info);
    if (st != B2P_OK) return st;
    Ctx* ctx = new (std::nothrow) Ctx();
    if (!ctx) return B2P_OUT_OF_MEMORY;
    ctx->device = device;
    ctx->sm_count = info.multiprocessor_count;
    ctx->l2_bytes = info.l2_cache_bytes;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        delete ctx;
        return B2P_GPU_UNAVAILABLE;
    }
    ctx->stream = ctx->own_stream;
    *ctx_out = ctx;
    return B2P_OK;
}

int b2p_ctx_set_stream(void* p, void* stream) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    cudaSetDevice(ctx->device);
    B2P_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return B2P_OK;
}

int b2p_kernel_timing(void* p, const b2p_params* params, int reps, double* primal_ms, double* dual_ms,
                      double* primal_bytes, double* dual_bytes) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (!ctx->has_lp || !ctx->hw) {
        ctx->err = "b2p_kernel_timing: solve an uploaded LP with the Halpern engine first";
        return B2P_NO_LP;
    }
    if (!params || reps <= 0) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    return halpern_kernel_timing(ctx, params, reps, primal_ms, dual_ms, primal_bytes, dual_bytes);
}

int b2p_ctx_destroy(void* p) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    halpern_free(ctx);
    batch_free(ctx);
    mlp_free(ctx);
    ctx->lp.~DevLP();
    new (&ctx->lp) DevLP();
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return B2P_OK;
}

const char* b2p_last_error(void* p) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

// ---- GpuBackend::spmv (gpu_backend.cpp:34-86): INVALID_ARGUMENT on an empty matrix or missing x.
int b2p_spmv(void* p, int m, int n, const int32_t* rowptr, const int32_t* colidx, const double* vals,
             const double* x, double* y, b2p_timing_t* timing) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (m <= 0 || n <= 0 || !rowptr || !x || !y) return B2P_INVALID_ARGUMENT;
    int64_t nnz = rowptr[m];
    if (nnz > 0 && (!colidx || !vals)) return B2P_INVALID_ARGUMENT;
    if (!host_rowptr_ok(m, nnz, rowptr)) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    double t0 = now_ms();
    PhaseTimer pt;
    cudaStream_t s = ctx->stream;
    B2P_CUDA(ctx, ctx->s_rowptr.reserve(m + 1));
    B2P_CUDA(ctx, ctx->s_colidx.reserve(nnz));
    B2P_CUDA(ctx, ctx->s_vals.reserve(nnz));
    B2P_CUDA(ctx, ctx->s_x.reserve(n));
    B2P_CUDA(ctx, ctx->s_y.reserve(m));
    B2P_CUDA(ctx, ctx->s_flag.reserve(1));
    cudaEventRecord(pt.e[0], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_rowptr.p, rowptr, sizeof(int32_t) * (m + 1), cudaMemcpyHostToDevice, s));
    if (nnz) {
        B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_colidx.p, colidx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_vals.p, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_x.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemsetAsync(ctx->s_flag.p, 0, sizeof(int32_t), s));
    cudaEventRecord(pt.e[1], s);
    unsigned g = grid_for(m, 256, ctx->sm_count);
    k_validate_csr<<<g, 256, 0, s>>>(m, n, ctx->s_rowptr.p, ctx->s_colidx.p, ctx->s_flag.p);
    k_spmv_f64<<<g, 256, 0, s>>>(m, ctx->s_rowptr.p, ctx->s_colidx.p, ctx->s_vals.p, ctx->s_x.p, ctx->s_y.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    cudaEventRecord(pt.e[2], s);
    int32_t bad = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(y, ctx->s_y.p, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(&bad, ctx->s_flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pt.e[3], s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    pt.fill(timing, t0);
    if (bad) {
        ctx->err = "CSR column indices out of range or not strictly ascending in row " + std::to_string(bad - 1);
        return B2P_INVALID_ARGUMENT;
    }
    return B2P_OK;
}

// A^T y with the transpose built on the device; the sum over each column runs in
// ascending row order, as the reference scatter (src/sparse_matrix.cpp:175-185) does.
int b2p_spmv_t(void* p, int m, int n, const int32_t* rowptr, const int32_t* colidx, const double* vals,
               const double* yv, double* w, b2p_timing_t* timing) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (m <= 0 || n <= 0 || !rowptr || !yv || !w) return B2P_INVALID_ARGUMENT;
    int64_t nnz = rowptr[m];
    if (nnz > 0 && (!colidx || !vals)) return B2P_INVALID_ARGUMENT;
    if (!host_rowptr_ok(m, nnz, rowptr)) return B2P_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    double t0 = now_ms();
    PhaseTimer pt;
    cudaStream_t s = ctx->stream;
    DBuf<int32_t> rp, ci, trp, tci;
    DBuf<double> va, tva;
    B2P_CUDA(ctx, rp.reserve(m + 1));
    B2P_CUDA(ctx, ci.reserve(nnz));
    B2P_CUDA(ctx, va.reserve(nnz));
    B2P_CUDA(ctx, trp.reserve(n + 1));
    B2P_CUDA(ctx, tci.reserve(nnz));
    B2P_CUDA(ctx, tva.reserve(nnz));
    B2P_CUDA(ctx, ctx->s_x.reserve(m));
    B2P_CUDA(ctx, ctx->s_y.reserve(n));
    B2P_CUDA(ctx, ctx->s_flag.reserve(1));
    cudaEventRecord(pt.e[0], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(rp.p, rowptr, sizeof(int32_t) * (m + 1), cudaMemcpyHostToDevice, s));
    if (nnz) {
        B2P_CUDA(ctx, cudaMemcpyAsync(ci.p, colidx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(va.p, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_x.p, yv, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemsetAsync(ctx->s_flag.p, 0, sizeof(int32_t), s));
    cudaEventRecord(pt.e[1], s);
    unsigned g = grid_for(m, 256, ctx->sm_count);
    k_validate_csr<<<g, 256, 0, s>>>(m, n, rp.p, ci.p, ctx->s_flag.p);
    int32_t bad = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&bad, ctx->s_flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    if (bad) {
        ctx->err = "CSR column indices out of range or not strictly ascending in row " + std::to_string(bad - 1);
        return B2P_INVALID_ARGUMENT;
    }
    int st = build_transpose(ctx, m, n, nnz, rp.p, ci.p, va.p, trp.p, tci.p, tva.p);
    if (st) return st;
    unsigned gn = grid_for(n, 256, ctx->sm_count);
    k_spmv_f64<<<gn, 256, 0, s>>>(n, trp.p, tci.p, tva.p, ctx->s_x.p, ctx->s_y.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    cudaEventRecord(pt.e[2], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(w, ctx->s_y.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pt.e[3], s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    pt.fill(timing, t0);
    return B2P_OK;
}

int b2p_vector_op(void* p, int op, size_t n, double alpha, const double* a, const double* bv, double* out,
                  b2p_timing_t* timing) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (op < 0 || op > 3 || !a || !out) return B2P_INVALID_ARGUMENT;
    bool needs_b = (op != B2P_VEC_SCALE);
    if (needs_b && !bv) return B2P_INVALID_ARGUMENT;
    if (n == 0) return B2P_OK;
    cudaSetDevice(ctx->device);
    double t0 = now_ms();
    PhaseTimer pt;
    cudaStream_t s = ctx->stream;
    B2P_CUDA(ctx, ctx->s_x.reserve(n));
    B2P_CUDA(ctx, ctx->s_y.reserve(n));
    B2P_CUDA(ctx, ctx->s_z.reserve(n));
    cudaEventRecord(pt.e[0], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_x.p, a, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (needs_b) B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_y.p, bv, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    cudaEventRecord(pt.e[1], s);
    k_vec<<<grid_for((int64_t)n, 256, ctx->sm_count), 256, 0, s>>>(op, n, alpha, ctx->s_x.p, ctx->s_y.p, ctx->s_z.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    cudaEventRecord(pt.e[2], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(out, ctx->s_z.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pt.e[3], s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    pt.fill(timing, t0);
    return B2P_OK;
}

static int dot_impl(Ctx* ctx, size_t n, const double* a, const double* bv, double* out, b2p_timing_t* timing,
                    bool sqrt_out) {
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (!a || !out) return B2P_INVALID_ARGUMENT;
    if (n == 0) {
        *out = 0.0;
        return B2P_OK;
    }
    cudaSetDevice(ctx->device);
    double t0 = now_ms();
    PhaseTimer pt;
    cudaStream_t s = ctx->stream;
    B2P_CUDA(ctx, ctx->s_x.reserve(n));
    B2P_CUDA(ctx, ctx->s_y.reserve(n));
    B2P_CUDA(ctx, ctx->s_z.reserve(kRedBlocks + 1));
    cudaEventRecord(pt.e[0], s);
    B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_x.p, a, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (bv) B2P_CUDA(ctx, cudaMemcpyAsync(ctx->s_y.p, bv, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    cudaEventRecord(pt.e[1], s);
    k_dot_partial<<<kRedBlocks, kRedThreads, 0, s>>>(n, ctx->s_x.p, bv ? ctx->s_y.p : nullptr, ctx->s_z.p);
    k_sum_partials<<<1, kRedThreads, 0, s>>>(kRedBlocks, ctx->s_z.p, ctx->s_z.p + kRedBlocks);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    cudaEventRecord(pt.e[2], s);
    double r = 0.0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&r, ctx->s_z.p + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    cudaEventRecord(pt.e[3], s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    pt.fill(timing, t0);
    *out = sqrt_out ? std::sqrt(r) : r;
    return B2P_OK;
}

int b2p_dot(void* p, size_t n, const double* a, const double* b, double* out, b2p_timing_t* timing) {
    if (!b) return B2P_INVALID_ARGUMENT;
    return dot_impl(as_ctx(p), n, a, b, out, timing, false);
}

int b2p_norm2(void* p, size_t n, const double* a, double* out, b2p_timing_t* timing) {
    return dot_impl(as_ctx(p), n, a, nullptr, out, timing, true);
}

// ---- single LP upload
int b2p_upload_lp(void* p, int m, int n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx,
                  const double* vals, const double* b, const double* c, const double* lb, const double* ub,
                  const uint8_t* is_eq) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (m <= 0 || n <= 0 || nnz < 0 || nnz > INT32_MAX || !rowptr || !b || !c || !lb || !ub || !is_eq) {
        ctx->err = "b2p_upload_lp: empty LP or null argument";
        return B2P_INVALID_ARGUMENT;
    }
    if (nnz > 0 && (!colidx || !vals)) return B2P_INVALID_ARGUMENT;
    if (!host_rowptr_ok(m, nnz, rowptr)) {
        ctx->err = "b2p_upload_lp: row pointer array is not a valid CSR offset array";
        return B2P_INVALID_ARGUMENT;
    }
    for (int j = 0; j < n; ++j) {
        if (std::isnan(lb[j]) || std::isnan(ub[j]) || std::isnan(c[j])) {
            ctx->err = "b2p_upload_lp: NaN in c / lb / ub";
            return B2P_INVALID_ARGUMENT;
        }
    }
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    ctx->has_lp = false;
    DevLP& L = ctx->lp;
    L.m = m;
    L.n = n;
    L.nnz = nnz;
    B2P_CUDA(ctx, L.rowptr.reserve(m + 1));
    B2P_CUDA(ctx, L.colidx.reserve(nnz));
    B2P_CUDA(ctx, L.vals.reserve(nnz));
    B2P_CUDA(ctx, L.t_rowptr.reserve(n + 1));
    B2P_CUDA(ctx, L.t_colidx.reserve(nnz));
    B2P_CUDA(ctx, L.t_vals.reserve(nnz));
    B2P_CUDA(ctx, L.b.reserve(m));
    B2P_CUDA(ctx, L.c.reserve(n));
    B2P_CUDA(ctx, L.lb.reserve(n));
    B2P_CUDA(ctx, L.ub.reserve(n));
    B2P_CUDA(ctx, L.is_eq.reserve(m));
    B2P_CUDA(ctx, ctx->s_flag.reserve(1));
    B2P_CUDA(ctx, cudaMemcpyAsync(L.rowptr.p, rowptr, sizeof(int32_t) * (m + 1), cudaMemcpyHostToDevice, s));
    if (nnz) {
        B2P_CUDA(ctx, cudaMemcpyAsync(L.colidx.p, colidx, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(L.vals.p, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    }
    B2P_CUDA(ctx, cudaMemcpyAsync(L.b.p, b, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(L.c.p, c, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(L.lb.p, lb, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(L.ub.p, ub, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(L.is_eq.p, is_eq, m, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemsetAsync(ctx->s_flag.p, 0, sizeof(int32_t), s));
    k_validate_csr<<<grid_for(m, 256, ctx->sm_count), 256, 0, s>>>(m, n, L.rowptr.p, L.colidx.p, ctx->s_flag.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    int32_t bad = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(&bad, ctx->s_flag.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    if (bad) {
        ctx->err = "b2p_upload_lp: column indices out of range or not strictly ascending in row " + std::to_string(bad - 1);
        return B2P_INVALID_ARGUMENT;
    }
    int st = build_transpose(ctx, m, n, nnz, L.rowptr.p, L.colidx.p, L.vals.p, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p);
    if (st) return st;
    double bn = 0, cn = 0;
    for (int i = 0; i < m; ++i) bn += b[i] * b[i];
    for (int j = 0; j < n; ++j) cn += c[j] * c[j];
    L.bnorm = std::sqrt(bn);
    L.cnorm = std::sqrt(cn);
    L.mean_row_len = (double)nnz / m;
    L.mean_col_len = (double)nnz / n;
    int mr = 0;
    for (int i = 0; i < m; ++i) mr = std::max(mr, rowptr[i + 1] - rowptr[i]);
    L.max_row_len = mr;
    ctx->lp_gen += 1;
    ctx->has_lp = true;
    return B2P_OK;
}

int b2p_solve(void* p, const b2p_params* params, const double* x0, const double* y0, b2p_result* result,
              double* x_out, double* y_out) {
    Ctx* ctx = as_ctx(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (!result) return B2P_INVALID_ARGUMENT;
    if (!ctx->has_lp) {
        ctx->err = "b2p_solve: no LP uploaded";
        return B2P_NO_LP;
    }
    b2p_params def;
    b2p_params_default(&def);
    const b2p_params* pp = params ? params : &def;
    std::memset(result, 0, sizeof(*result));
    if (pp->max_iterations < 0 || pp->check_frequency <= 0 || pp->check_every <= 0) {
        ctx->err = "b2p_solve: max_iterations < 0 or non-positive check cadence";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    int64_t l0 = ctx->launches;
    double t0 = now_ms();
    int st;
    if (pp->engine == B2P_ENGINE_REFERENCE)
        st = ref_engine_solve(ctx, pp, result, x_out, y_out);
    else if (pp->engine == B2P_ENGINE_HALPERN)
        st = halpern_engine_solve(ctx, pp, x0, y0, result, x_out, y_out);
    else {
        ctx->err = "b2p_solve: unknown engine";
        return B2P_INVALID_ARGUMENT;
    }
    result->solve_time_ms = now_ms() - t0;
    result->kernel_launches = ctx->launches - l0;
    return st;
}

}  // extern "C"
