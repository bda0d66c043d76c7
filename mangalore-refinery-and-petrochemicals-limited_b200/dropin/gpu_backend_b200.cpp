// Drop-in replacement for the reference's src/gpu_backend.cpp.
//
// Implements every member of bharatopt::GpuBackend declared in the reference
// header include/bharatopt/gpu_backend.hpp:171-233 on top of libb2p:
//   initialize / device_info   -> b2p_device_info   (a real device query instead of a
//                                                     hard-coded, always-unavailable GPU)
//   spmv                       -> b2p_spmv           (FP64 CSR SpMV on the B200)
//   spmv_with_cpu_comparison   -> b2p_spmv + the reference's CSRMatrix::multiply
//   vector_add/_sub/_scale,axpy-> b2p_vector_op
//   dot_product / norm2        -> b2p_dot / b2p_norm2
// Argument checks and status codes are those of the reference members
// (src/gpu_backend.cpp:34-327); GpuBuffer stays the header-defined host-backed
// buffer, so each call stages its operands to the device and back.  Without a
// usable GPU every compute call returns GPUStatus::GPU_UNAVAILABLE -- there is
// no host fallback loop.
#include <bharatopt/gpu_backend.hpp>

#include <chrono>
#include <mutex>

#include "../../include/b2p.h"

namespace bharatopt {

namespace {

std::mutex g_ctx_mutex;
void* g_ctx = nullptr;

void* backend_context() {
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    if (!g_ctx) {
        void* c = nullptr;
        if (b2p_ctx_create(0, &c) == B2P_OK) g_ctx = c;
    }
    return g_ctx;
}

GPUStatus to_gpu_status(int st) {
    switch (st) {
        case B2P_OK: return GPUStatus::SUCCESS;
        case B2P_GPU_UNAVAILABLE: return GPUStatus::GPU_UNAVAILABLE;
        case B2P_GPU_UNINITIALIZED: return GPUStatus::GPU_UNINITIALIZED;
        case B2P_OUT_OF_MEMORY: return GPUStatus::OUT_OF_MEMORY;
        case B2P_INVALID_ARGUMENT: return GPUStatus::INVALID_ARGUMENT;
        default: return GPUStatus::EXECUTION_FAILED;
    }
}

void copy_timing(const b2p_timing_t& t, GpuTimingResult* out) {
    if (!out) return;
    out->h2d_time_ms = t.h2d_time_ms;
    out->kernel_time_ms = t.kernel_time_ms;
    out->d2h_time_ms = t.d2h_time_ms;
    out->sync_time_ms = t.sync_time_ms;
    out->total_gpu_time_ms = t.total_gpu_time_ms;
}

}  // namespace

// The device is probed when the singleton is first used, so is_available() is
// truthful for every caller -- including ProblemAnalyser::extract_features
// (src/cost_estimator.cpp:87-90), which reads it without calling initialize().
GpuBackend& GpuBackend::instance() {
    static GpuBackend backend;
    static const bool probed = (backend.initialize(), true);
    (void)probed;
    return backend;
}

GPUStatus GpuBackend::initialize() {
    if (initialized_) return device_info_.is_available ? GPUStatus::SUCCESS : GPUStatus::GPU_UNAVAILABLE;
    b2p_device_info_t info;
    int st = b2p_device_info(0, &info);
    device_info_.device_name = info.device_name;
    device_info_.total_memory_bytes = info.total_memory_bytes;
    device_info_.free_memory_bytes = info.free_memory_bytes;
    device_info_.compute_capability_major = info.compute_capability_major;
    device_info_.compute_capability_minor = info.compute_capability_minor;
    device_info_.status_message = info.status_message;
    device_info_.is_available = (st == B2P_OK) && backend_context() != nullptr;
    initialized_ = true;
    return device_info_.is_available ? GPUStatus::SUCCESS : GPUStatus::GPU_UNAVAILABLE;
}

GPUStatus GpuBackend::spmv(const GpuMatrixCSR& A, const GpuBuffer<real_t>& x, GpuBuffer<real_t>& y,
                           GpuTimingResult* timing) {
    if (!A.is_valid() || !x.is_allocated() || x.size() < A.cols) return GPUStatus::INVALID_ARGUMENT;
    if (y.size() < A.rows) {
        GPUStatus stat = y.allocate(A.rows);
        if (stat != GPUStatus::SUCCESS) return stat;
    }
    if (initialize() != GPUStatus::SUCCESS) return GPUStatus::GPU_UNAVAILABLE;
    b2p_timing_t t{};
    int st = b2p_spmv(backend_context(), (int)A.rows, (int)A.cols, A.row_offsets.data(),
                      A.nnz ? A.col_indices.data() : nullptr, A.nnz ? A.values.data() : nullptr, x.data(), y.data(), &t);
    copy_timing(t, timing);
    return to_gpu_status(st);
}

GPUStatus GpuBackend::spmv_with_cpu_comparison(const CSRMatrix& cpu_A, const std::vector<real_t>& cpu_x,
                                               std::vector<real_t>& gpu_y, real_t& max_abs_error,
                                               GpuTimingResult* timing) {
    if (!cpu_A.is_valid() || cpu_x.size() != cpu_A.cols()) return GPUStatus::INVALID_ARGUMENT;
    auto c0 = std::chrono::high_resolution_clock::now();
    std::vector<real_t> cpu_y = cpu_A.multiply(cpu_x);
    auto c1 = std::chrono::high_resolution_clock::now();
    GpuMatrixCSR gpu_A;
    GPUStatus s = gpu_A.upload_from_cpu(cpu_A);
    if (s != GPUStatus::SUCCESS) return s;
    GpuBuffer<real_t> gx(cpu_x.size());
    s = gx.copy_host_to_device(cpu_x.data(), cpu_x.size());
    if (s != GPUStatus::SUCCESS) return s;
    GpuBuffer<real_t> gy(cpu_A.rows());
    s = spmv(gpu_A, gx, gy, timing);
    if (s != GPUStatus::SUCCESS) return s;
    gpu_y.resize(cpu_A.rows());
    s = gy.copy_device_to_host(gpu_y.data(), cpu_A.rows());
    if (s != GPUStatus::SUCCESS) return s;
    max_abs_error = 0.0;
    for (size_t i = 0; i < cpu_A.rows(); ++i) {
        real_t d = std::abs(gpu_y[i] - cpu_y[i]);
        if (d > max_abs_error) max_abs_error = d;
    }
    if (timing) timing->cpu_reference_time_ms = std::chrono::duration<double, std::milli>(c1 - c0).count();
    return GPUStatus::SUCCESS;
}

namespace {

GPUStatus vec_op(GpuBackend& be, int op, real_t alpha, const GpuBuffer<real_t>& a, const GpuBuffer<real_t>* b,
                 GpuBuffer<real_t>& result, size_t n, GpuTimingResult* timing) {
    if (!a.is_allocated() || a.size() < n || (b && (!b->is_allocated() || b->size() < n)))
        return GPUStatus::INVALID_ARGUMENT;
    if (result.size() < n) {
        GPUStatus stat = result.allocate(n);
        if (stat != GPUStatus::SUCCESS) return stat;
    }
    if (be.initialize() != GPUStatus::SUCCESS) return GPUStatus::GPU_UNAVAILABLE;
    b2p_timing_t t{};
    int st = b2p_vector_op(backend_context(), op, n, alpha, a.data(), b ? b->data() : nullptr, result.data(), &t);
    copy_timing(t, timing);
    return to_gpu_status(st);
}

}  // namespace

GPUStatus GpuBackend::vector_add(const GpuBuffer<real_t>& a, const GpuBuffer<real_t>& b, GpuBuffer<real_t>& result,
                                 size_t n, GpuTimingResult* timing) {
    return vec_op(*this, B2P_VEC_ADD, 0.0, a, &b, result, n, timing);
}

GPUStatus GpuBackend::vector_sub(const GpuBuffer<real_t>& a, const GpuBuffer<real_t>& b, GpuBuffer<real_t>& result,
                                 size_t n, GpuTimingResult* timing) {
    return vec_op(*this, B2P_VEC_SUB, 0.0, a, &b, result, n, timing);
}

GPUStatus GpuBackend::vector_scale(const GpuBuffer<real_t>& input, real_t alpha, GpuBuffer<real_t>& result, size_t n,
                                   GpuTimingResult* timing) {
    return vec_op(*this, B2P_VEC_SCALE, alpha, input, nullptr, result, n, timing);
}

GPUStatus GpuBackend::axpy(real_t alpha, const GpuBuffer<real_t>& x, const GpuBuffer<real_t>& y_in,
                           GpuBuffer<real_t>& y_out, size_t n, GpuTimingResult* timing) {
    return vec_op(*this, B2P_VEC_AXPY, alpha, x, &y_in, y_out, n, timing);
}

GPUStatus GpuBackend::dot_product(const GpuBuffer<real_t>& a, const GpuBuffer<real_t>& b, real_t& result, size_t n,
                                  GpuTimingResult* timing) {
    if (!a.is_allocated() || !b.is_allocated() || a.size() < n || b.size() < n) return GPUStatus::INVALID_ARGUMENT;
    if (initialize() != GPUStatus::SUCCESS) return GPUStatus::GPU_UNAVAILABLE;
    b2p_timing_t t{};
    int st = b2p_dot(backend_context(), n, a.data(), b.data(), &result, &t);
    copy_timing(t, timing);
    return to_gpu_status(st);
}

GPUStatus GpuBackend::norm2(const GpuBuffer<real_t>& v, real_t& result, size_t n, GpuTimingResult* timing) {
    if (!v.is_allocated() || v.size() < n) return GPUStatus::INVALID_ARGUMENT;
    if (initialize() != GPUStatus::SUCCESS) return GPUStatus::GPU_UNAVAILABLE;
    b2p_timing_t t{};
    int st = b2p_norm2(backend_context(), n, v.data(), &result, &t);
    copy_timing(t, timing);
    return to_gpu_status(st);
}

}  // namespace bharatopt
