// Reference engine: the reference PDHG (CPUFirstOrderSolver::solve,
// src/first_order_solver.cpp:103-279) on the GPU, iterate for iterate.
//
// Compiled with --fmad=false and with every sum taken in the reference's order
// (rows ascending inside each column for A^T y, columns ascending inside each
// row for A x), so x^k, y^k, the convergence checks, the iteration count and
// the status are bit-identical to the compiled reference.
//
// Layout: one thread per column (primal step over the CSR of A^T) and one
// thread per row (dual step over the CSR of A).  The check_frequency
// iterations between two convergence checks are captured once as a CUDA graph
// (2 kernels per iteration + 2 check kernels) and replayed; the host reads back
// four doubles per check.
#include <cmath>
#include <cstring>

#include "b2p_internal.cuh"

namespace b2p {

namespace {

// bharatopt::clamp (include/bharatopt/config.hpp:25-28): NaN passes through.
__device__ __forceinline__ double ref_clamp(double v, double lo, double hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}

// Slots of the per-check reduction block.
enum { R_DPRIMAL = 0, R_DDUAL, R_VIOL_X, R_VIOL_AVG, R_BOUND, R_COUNT };

struct RefState {
    double *tau, *sigma, *x, *y, *x_hat, *x_sum, *x_avg;
    unsigned long long* red;  // R_COUNT slots (bit patterns of non-negative doubles)
    long long* iter;          // device iteration counter (== avg_count)
};

// first_order_solver.cpp:103-128
__global__ void k_ref_steps(int m, int n, const int32_t* __restrict__ rowptr, const double* __restrict__ vals,
                            const int32_t* __restrict__ t_rowptr, const double* __restrict__ t_vals, int adaptive,
                            double pstep, double dstep, double* __restrict__ tau, double* __restrict__ sigma) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += stride) {
        double s = 0.0;
        for (int k = t_rowptr[j]; k < t_rowptr[j + 1]; ++k) s += fabs(t_vals[k]);
        tau[j] = adaptive ? ((s > 1e-12) ? (0.95 / s) : 1.0) : pstep;
    }
    for (int i = tid; i < m; i += stride) {
        double s = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) s += fabs(vals[k]);
        sigma[i] = adaptive ? ((s > 1e-12) ? (0.95 / s) : 1.0) : dstep;
    }
}

// first_order_solver.cpp:130-151
__global__ void k_ref_init(int m, int n, const double* __restrict__ lb, const double* __restrict__ ub,
                           double* __restrict__ x, double* __restrict__ y, double* __restrict__ x_sum,
                           long long* iter, unsigned long long* red) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const double inf = INFINITY;
    for (int j = tid; j < n; j += stride) {
        double target = 0.0;
        if (lb[j] > -inf && ub[j] < inf) target = 0.5 * (lb[j] + ub[j]);
        else if (lb[j] > -inf) target = lb[j];
        else if (ub[j] < inf) target = ub[j];
        x[j] = ref_clamp(target, lb[j], ub[j]);
        x_sum[j] = 0.0;
    }
    for (int i = tid; i < m; i += stride) y[i] = 0.0;
    if (tid == 0) {
        *iter = 0;
        for (int r = 0; r < R_COUNT; ++r) red[r] = 0ull;
    }
}

// Steps A-C (first_order_solver.cpp:163-180): A^T y, projected primal step,
// ergodic sum, extrapolation.  x_prev == x at entry, so x_hat = 2 x_new - x.
template <bool CHECK>
__global__ void __launch_bounds__(256) k_ref_primal(int n, const int32_t* __restrict__ t_rowptr,
                                                    const int32_t* __restrict__ t_colidx,
                                                    const double* __restrict__ t_vals, const double* __restrict__ c,
                                                    const double* __restrict__ lb, const double* __restrict__ ub,
                                                    RefState st) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double w = 0.0;
        for (int k = t_rowptr[j]; k < t_rowptr[j + 1]; ++k) w += t_vals[k] * st.y[t_colidx[k]];
        double xj = st.x[j];
        double grad = c[j] + w;
        double next_x = xj - st.tau[j] * grad;
        double new_x = ref_clamp(next_x, lb[j], ub[j]);
        if (CHECK) atomic_max_nonneg(&st.red[R_DPRIMAL], fabs(new_x - xj));
        st.x_sum[j] += new_x;
        st.x_hat[j] = 2.0 * new_x - xj;
        st.x[j] = new_x;
    }
}

// Steps D-E (first_order_solver.cpp:183-192): A x_hat, dual step, sign projection.
template <bool CHECK>
__global__ void __launch_bounds__(256) k_ref_dual(int m, const int32_t* __restrict__ rowptr,
                                                  const int32_t* __restrict__ colidx, const double* __restrict__ vals,
                                                  const double* __restrict__ b, const uint8_t* __restrict__ is_eq,
                                                  RefState st) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = tid; i < m; i += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) v += vals[k] * st.x_hat[colidx[k]];
        double yi = st.y[i];
        double next_y = yi + st.sigma[i] * (v - b[i]);
        // std::max(0.0, next_y) == (0.0 < next_y) ? next_y : 0.0
        double new_y = (!is_eq[i]) ? ((0.0 < next_y) ? next_y : 0.0) : next_y;
        if (CHECK) atomic_max_nonneg(&st.red[R_DDUAL], fabs(new_y - yi));
        st.y[i] = new_y;
    }
    if (tid == 0) *st.iter += 1;
}

// Step F, column part (first_order_solver.cpp:208-218): bound violation of x and the
// clamped ergodic average x_avg = clamp(x_sum / avg_count).
__global__ void k_ref_check_cols(int n, const double* __restrict__ lb, const double* __restrict__ ub, RefState st) {
    long long cnt = *st.iter;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double xj = st.x[j];
        if (xj < lb[j] - 1e-12) atomic_max_nonneg(&st.red[R_BOUND], lb[j] - xj);
        if (xj > ub[j] + 1e-12) atomic_max_nonneg(&st.red[R_BOUND], xj - ub[j]);
        st.x_avg[j] = (cnt > 0) ? ref_clamp(st.x_sum[j] / (double)cnt, lb[j], ub[j]) : xj;
    }
}

// Step F, row part (first_order_solver.cpp:199-206, 219-225): max row violation of x and x_avg.
__global__ void k_ref_check_rows(int m, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                                 const double* __restrict__ vals, const double* __restrict__ b,
                                 const uint8_t* __restrict__ is_eq, RefState st) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double ax = 0.0, aa = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) ax += vals[k] * st.x[colidx[k]];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) aa += vals[k] * st.x_avg[colidx[k]];
        double d1 = ax - b[i], d2 = aa - b[i];
        double v1 = (!is_eq[i]) ? ((0.0 < d1) ? d1 : 0.0) : fabs(d1);
        double v2 = (!is_eq[i]) ? ((0.0 < d2) ? d2 : 0.0) : fabs(d2);
        atomic_max_nonneg(&st.red[R_VIOL_X], v1);
        atomic_max_nonneg(&st.red[R_VIOL_AVG], v2);
    }
}

__global__ void k_ref_clear(unsigned long long* red) {
    if (threadIdx.x < R_COUNT) red[threadIdx.x] = 0ull;
}

double bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}

struct RefBuffers {
    DBuf<double> tau, sigma, x, y, x_hat, x_sum, x_avg;
    DBuf<unsigned long long> red;
    DBuf<long long> iter;
};

}  // namespace

int ref_engine_solve(Ctx* ctx, const b2p_params* p, b2p_result* r, double* x_out, double* y_out) {
    DevLP& L = ctx->lp;
    const int m = L.m, n = L.n;
    cudaStream_t s = ctx->stream;
    RefBuffers B;
    B2P_CUDA(ctx, B.tau.reserve(n));
    B2P_CUDA(ctx, B.sigma.reserve(m));
    B2P_CUDA(ctx, B.x.reserve(n));
    B2P_CUDA(ctx, B.y.reserve(m));
    B2P_CUDA(ctx, B.x_hat.reserve(n));
    B2P_CUDA(ctx, B.x_sum.reserve(n));
    B2P_CUDA(ctx, B.x_avg.reserve(n));
    B2P_CUDA(ctx, B.red.reserve(R_COUNT));
    B2P_CUDA(ctx, B.iter.reserve(1));
    RefState st{B.tau.p, B.sigma.p, B.x.p, B.y.p, B.x_hat.p, B.x_sum.p, B.x_avg.p, B.red.p, B.iter.p};

    const int TB = 256;
    unsigned gn = grid_for(n, TB, ctx->sm_count), gm = grid_for(m, TB, ctx->sm_count);
    unsigned gmn = grid_for(std::max(m, n), TB, ctx->sm_count);
    k_ref_steps<<<gmn, TB, 0, s>>>(m, n, L.rowptr.p, L.vals.p, L.t_rowptr.p, L.t_vals.p, p->adaptive_step_size,
                                   p->primal_step_size, p->dual_step_size, st.tau, st.sigma);
    k_ref_init<<<gmn, TB, 0, s>>>(m, n, L.lb.p, L.ub.p, st.x, st.y, st.x_sum, st.iter, st.red);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;

    auto plain_iter = [&]() {
        k_ref_primal<false><<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p, L.c.p, L.lb.p, L.ub.p, st);
        k_ref_dual<false><<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, L.b.p, L.is_eq.p, st);
    };
    auto check_iter = [&]() {
        k_ref_clear<<<1, 32, 0, s>>>(st.red);
        k_ref_primal<true><<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p, L.c.p, L.lb.p, L.ub.p, st);
        k_ref_dual<true><<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, L.b.p, L.is_eq.p, st);
        k_ref_check_cols<<<gn, TB, 0, s>>>(n, L.lb.p, L.ub.p, st);
        k_ref_check_rows<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, L.b.p, L.is_eq.p, st);
    };

    const int64_t max_it = p->max_iterations;
    const int64_t cf = std::min<int64_t>(p->check_frequency, 100);  // first_order_solver.cpp:156
    // One check interval = cf-1 plain iterations + 1 check iteration, captured once.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (max_it >= cf) {
        B2P_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int64_t k = 0; k < cf - 1; ++k) plain_iter();
        check_iter();
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (ce != cudaSuccess) {
            ctx->err = std::string("graph capture: ") + cudaGetErrorString(ce);
            return B2P_EXECUTION_FAILED;
        }
        B2P_CUDA(ctx, cudaGraphInstantiate(&exec, graph, 0));
    }
    struct GraphGuard {
        cudaGraph_t g;
        cudaGraphExec_t e;
        ~GraphGuard() {
            if (e) cudaGraphExecDestroy(e);
            if (g) cudaGraphDestroy(g);
        }
    } guard{graph, exec};

    unsigned long long host_red[R_COUNT];
    int64_t iter = 0;
    bool converged = false, failed = false;
    double cons_viol = 0.0, bound_viol = 0.0, dpr = 0.0, ddu = 0.0;
    cudaEventRecord(ctx->ev0, s);
    while (iter < max_it) {
        int64_t next_check = std::min<int64_t>((iter / cf + 1) * cf, max_it);
        int64_t span = next_check - iter;
        if (span == cf && exec) {
            B2P_CUDA(ctx, cudaGraphLaunch(exec, s));
            ctx->launches += 2 * cf + 3;
        } else {
            for (int64_t k = 0; k < span - 1; ++k) plain_iter();
            check_iter();
            B2P_LAUNCH(ctx);
            ctx->launches += 2 * span + 3;
        }
        iter = next_check;
        B2P_CUDA(ctx, cudaMemcpyAsync(host_red, st.red, sizeof(host_red), cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        double vx = bits_to_double(host_red[R_VIOL_X]), va = bits_to_double(host_red[R_VIOL_AVG]);
        double best = (va < vx) ? va : vx;  // std::min(max_viol, avg_viol)
        bound_viol = bits_to_double(host_red[R_BOUND]);
        dpr = bits_to_double(host_red[R_DPRIMAL]);
        ddu = bits_to_double(host_red[R_DDUAL]);
        cons_viol = best;
        if (std::isnan(best) || best > 1e15) {  // first_order_solver.cpp:232-236
            failed = true;
            break;
        }
        bool feasible = best <= p->feasibility_tolerance && bound_viol <= p->feasibility_tolerance;
        bool stationary = dpr <= 1e-7 && ddu <= 1e-7;
        if (feasible && stationary && iter >= 100) {
            converged = true;
            break;
        }
    }
    cudaEventRecord(ctx->ev1, s);
    r->iterations = iter;
    r->constraint_violation = cons_viol;
    r->bound_violation = bound_viol;
    r->max_primal_delta = dpr;
    r->max_dual_delta = ddu;
    if (failed) {
        r->status = B2P_STATUS_NUMERICAL_FAILURE;
    } else {
        r->status = converged ? B2P_STATUS_OPTIMAL : B2P_STATUS_MAX_ITERATIONS;
        // first_order_solver.cpp:261-279: the ergodic average replaces x only when the
        // loop did not converge and its violation is no worse than the last check's.
        k_ref_clear<<<1, 32, 0, s>>>(st.red);
        k_ref_check_cols<<<gn, TB, 0, s>>>(n, L.lb.p, L.ub.p, st);
        k_ref_check_rows<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, L.b.p, L.is_eq.p, st);
        B2P_LAUNCH(ctx);
        ctx->launches += 3;
        B2P_CUDA(ctx, cudaMemcpyAsync(host_red, st.red, sizeof(host_red), cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        double avg_viol = bits_to_double(host_red[R_VIOL_AVG]);
        r->used_average = (!converged && avg_viol <= cons_viol) ? 1 : 0;
    }
    float kms = 0.f;
    cudaEventElapsedTime(&kms, ctx->ev0, ctx->ev1);
    r->kernel_time_ms = kms;
    double t0 = now_ms();
    if (x_out) B2P_CUDA(ctx, cudaMemcpyAsync(x_out, r->used_average ? st.x_avg : st.x, sizeof(double) * n,
                                             cudaMemcpyDeviceToHost, s));
    if (y_out) B2P_CUDA(ctx, cudaMemcpyAsync(y_out, st.y, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    r->transfer_time_ms = now_ms() - t0;
    return B2P_OK;
}

}  // namespace b2p
