// Allocation-free FP64 dot product: b2p_dot_noalloc.
//
// Who needs this: callers that must not allocate device memory themselves or
// have a library do it for them -- for example code that runs while a CUDA
// stream is being captured into a graph (cudaMalloc is not a legal operation
// there in the default capture mode), or an application that hands out all of
// its device memory from its own pool and treats a stray cudaMalloc (which can
// also synchronise the device) as a bug.  Such a caller owns the input and
// output buffers; everything else this entry point needs lives in a fixed
// scratch array below that the library reserves once, at load time.
//
// The computation is the same deterministic two-pass reduction as b2p_dot
// (b2p_api.cu): pass 1 writes one partial sum per block into the scratch array,
// pass 2 adds the partials in index order with one block.
#include <mutex>

#include "b2p_internal.cuh"

namespace b2p {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaItems = 8;  // elements per thread in pass 1
constexpr int kNaMaxPartials = B2P_DOT_NOALLOC_MAX_N / (kNaThreads * kNaItems);
static_assert(kNaMaxPartials * kNaThreads * kNaItems == B2P_DOT_NOALLOC_MAX_N, "max n must tile the scratch");

// One partial sum per pass-1 block: kNaMaxPartials doubles (32 KiB).  Every GPU
// that loads libb2p.so holds this array until the process exits.  All calls
// share it; it keeps whatever the last call wrote.
static __device__ __align__(256) double g_dot_scratch[kNaMaxPartials];

// Device address of g_dot_scratch on each device, looked up once per device.
// In host code the name g_dot_scratch is only a host-side stand-in for the
// array, not its device address, so kernels are always given this pointer.
std::mutex g_setup_mutex;
double* g_scratch_addr[64] = {nullptr};

__global__ void __launch_bounds__(kNaThreads) k_na_partials(size_t n, const double* __restrict__ a,
                                                             const double* __restrict__ b, double* __restrict__ partial) {
    __shared__ double sh[kNaThreads / 32];
    const size_t base = (size_t)blockIdx.x * kNaThreads * kNaItems;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kNaItems; ++q) {
        const size_t i = base + (size_t)q * kNaThreads + threadIdx.x;
        if (i < n) s += a[i] * b[i];
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kNaThreads / 32; ++w) t += sh[w];
        partial[blockIdx.x] = t;  // every partial this call reads is written by this call
    }
}

__global__ void __launch_bounds__(kNaThreads) k_na_sum(int count, const double* __restrict__ partial,
                                                        double* __restrict__ out) {
    __shared__ double sh[kNaThreads / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += kNaThreads) s += partial[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kNaThreads / 32; ++w) t += sh[w];
        *out = t;
    }
}

// Set-up for the current device: resolve the scratch array's device address once,
// and load both kernels onto the device (with lazy module loading a kernel is
// otherwise loaded at its first launch, which could then fall inside a later stream
// capture -- a first call with n == 0 never launches k_na_partials).  The cache is
// per device ordinal and is not invalidated: cudaDeviceReset is not supported.
int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return B2P_GPU_UNAVAILABLE;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_dot_scratch);
        if (e != cudaSuccess || !ptr) return map_cuda_error(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k_na_partials);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_na_sum);
        if (e != cudaSuccess) return map_cuda_error(e);
        g_scratch_addr[dev] = static_cast<double*>(ptr);
    }
    *out = g_scratch_addr[dev];
    return B2P_OK;
}

}  // namespace
}  // namespace b2p

extern "C" int b2p_dot_noalloc(const double* a_dev, const double* b_dev, size_t n, double* out_dev, void* stream) {
    using namespace b2p;
    if (!a_dev || !b_dev || !out_dev) return B2P_INVALID_ARGUMENT;
    if (n > (size_t)B2P_DOT_NOALLOC_MAX_N) return B2P_TOO_LARGE;
    double* scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st != B2P_OK) return st;
    // an error left pending by earlier, unrelated work is reported (not cleared) and
    // nothing is launched, so the status after the launches is this call's own
    cudaError_t pre = cudaPeekAtLastError();
    if (pre != cudaSuccess) return map_cuda_error(pre);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = n == 0 ? 0 : (int)((n + (size_t)kNaThreads * kNaItems - 1) / ((size_t)kNaThreads * kNaItems));
    if (blocks > 0) k_na_partials<<<blocks, kNaThreads, 0, s>>>(n, a_dev, b_dev, scratch);
    k_na_sum<<<1, kNaThreads, 0, s>>>(blocks, scratch, out_dev);  // blocks == 0 writes 0.0
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? B2P_OK : map_cuda_error(e);
}
