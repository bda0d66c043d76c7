// Halpern engine: restarted Halpern PDHG with reflection on a diagonally scaled LP.
//
// Precision: B2P_FP64 keeps everything in FP64.  B2P_FP32 (mixed) runs the
// iteration in FP32 -- scaled matrix values, the Halpern iterates x, y, their
// anchors and T(z), the problem vectors c, l, u, b and the dual bound, the SpMV
// sums and the vector updates -- while FP64 is kept for the Ruiz / Pock-Chambolle
// scaling factors, the squared-residual reductions that drive restarts, the KKT of
// the original LP, and the iterative refinement: at every restart the LP is
// re-centred on the current point (exact FP64 residuals b - A x, c + A^T y from
// the original matrix), so the FP32 iterates only ever carry a correction.
//
// Problem (standard form of src/first_order_solver.cpp:68-101):
//   min c.x  s.t. (Ax)_i <= b_i (<= rows) / = b_i (= rows),  l <= x <= u,
// Lagrangian c.x + y.(Ax - b), y >= 0 on <= rows (first_order_solver.cpp:185-192).
//
// Algorithm (Lu & Yang 2024, restarted Halpern PDHG; Ruiz / Pock-Chambolle
// scaling and primal-weight smoothing as in PDLP, Applegate et al. 2021):
//   T(x,y):  x~ = P_[l,u](x - tau (c + A^T y)),  xh = 2 x~ - x,
//            y~ = P_Y(y + sigma (A xh - b))
//   Halpern: z <- (k+1)/(k+2) ((1+rho) T(z) - rho z) + 1/(k+2) z_anchor
//   tau = eta/omega, sigma = eta*omega, eta = safety / ||A_s||_2
// Every `check_every` iterations (one chunk): fixed-point residual, FP64 KKT of
// T(z) on the ORIGINAL LP, restart test (sufficient / necessary / artificial),
// primal-weight update and termination -- all decided on the device by a
// one-thread control kernel, so a chunk is a fixed kernel sequence that is
// captured once as a CUDA graph and replayed until the control block says done.
//
// Kernels per iteration (HBM-bound; algorithmic bytes in kernel_timing_T below):
//   primal : A^T y + projected primal step + extrapolation + Halpern update
//            (+ check reductions)
//   dual   : A xh  + projected dual step + Halpern update (+ check reductions)
// each in one of three forms, picked per side by an autotuner on the uploaded LP:
//   k_iter_sell           SELL-32 copy of the operator (one lane per row, W-wide
//                         vector loads, no row pointers, no shuffles)
//   k_iter_sell<...,WIN>  the same, with each CTA's densest window of the gathered
//                         vector staged in shared memory
//   k_iter                CSR, L lanes per row, R rows per lane group
// The engine works on the LP renumbered so that rows and columns are sorted by
// length inside windows of 4096 (k_len_keys): the 32 rows of a SELL slice then have
// nearly equal lengths while rows that were neighbours stay near each other.
// Warm starts and answers are mapped between the caller's and the internal
// numbering on the device.
#include <cub/cub.cuh>

#include <cmath>
#include <cstring>
#include <algorithm>

#include "b2p_internal.cuh"

namespace b2p {

// Control block slots (device, FP64).
enum {
    A_RX2 = 0, A_RY2, A_RX2_FIRST, A_RY2_FIRST, A_DXA2, A_DYA2,   // restart residuals
    A_PRES2, A_DRES2, A_PC, A_BY, A_LAM,                          // KKT pieces
    A_EST,                                                        // sum |y| viol (objective-error bound)
    A_PRV2, A_PRC, A_PRM,           // primal ray dx: |viol|^2, c.dx, sum |c dx|
    A_DRB, A_DRL, A_DRM, A_DRV2,    // dual ray dy: b.dy, bound term of A^T dy, sum |terms|, |viol|^2
    A_COUNT
};

struct Ctrl {
    double acc[A_COUNT];
    double omega, eta, tau, sigma;
    double r0, rprev;
    double rel_p, rel_d, rel_g, pobj, dobj, obj_err;
    double eps, beta_s, beta_n, beta_a, bnorm, cnorm;
    double eps_obj, eps_inf;  // objective-accuracy stop, certificate tolerance (0 = off)
    // refinement: the solved (correction) problem maps back to the original LP as
    // x = xbar + pscale * dc * xt, y = ybar + dscale * dr * yt; the solve also stops
    // (status kInnerDone) once its fixed-point residual fell to inner_tol * r_first
    double pscale, dscale, inner_tol, r_first;
    long long k_base, total, max_iter, restarts;
    int K;
    int done, status, restart, first_after_restart;
};

// private status of a solve that reached its inner tolerance (refinement continues)
constexpr int kInnerDone = 100;

// SELL-32 copy of one orientation of the scaled matrix (internal numbering): slice s
// holds rows 32s..32s+31; its entries are stored in chunks of W per lane -- entry e
// of lane l sits at off[s] + (e / W) * 32 W + l W + e % W -- so one warp-wide
// load of W consecutive elements per lane reads 32 W contiguous elements.  Rows
// shorter than the slice's longest are zero-padded (value 0, index 0).
struct Sell {
    int C = 32;          // slice height (rows per slice): 32, 16 or 8
    int W = 1;
    int64_t slices = 0, total = 0;
    DBuf<int64_t> off;   // slices + 1
    DBuf<int32_t> idx;   // total
    DBuf<float> v32;     // total (mixed engine)
    DBuf<double> v64;    // total (FP64 engine)
    bool idx_ready = false;
};

// Per-CTA gather windows for one launch shape of a windowed SELL kernel.
struct Win {
    unsigned G = 0;      // grid (one resident wave)
    size_t smem = 0;     // dynamic shared memory per CTA (bytes); 0 = windows off
    DBuf<int32_t> lo, len;
};

struct HalpernWork {
    int m = -1, n = -1;
    // Internal numbering: rows and columns sorted by decreasing length inside
    // windows of kWindow, so that each 32-row slice of the SELL copies is nearly
    // uniform while neighbouring rows stay neighbours.  The engine works on `ilp`,
    // the uploaded LP renumbered; warm starts and answers are permuted on the device.
    int64_t ilp_gen = -1;        // ctx->lp_gen the internal copy was built from
    DevLP ilp;
    DBuf<int32_t> pr, pc;        // internal -> original row / column
    DBuf<int32_t> ic, ir;        // original -> internal column / row
    // SELL copies of A (rows) and A^T (columns), slice heights 32, 16, 8 (built on demand);
    // sr / sc point at the tuned one
    Sell sr_all[3], sc_all[3];
    Sell* sr = &sr_all[0];
    Sell* sc = &sc_all[0];
    bool sell_r = false, sell_c = false;  // tuned: SELL (true) or CSR kernel per side
    // tuned gather windows of the SELL kernels (smem 0 = none): grid, shared memory
    // bytes and the per-CTA windows built for that grid
    Win wr, wc;
    // tuned layout index (into sr_all / sc_all) and window shape (-1 = none) per side, so
    // a later upload of an LP of the same size can rebuild what the tuned shape needs
    int kr_t = 0, kc_t = 0, winr_t = -1, winc_t = -1;
    int64_t solved_gen = -1;     // upload generation and precision of the last solve
    int solved_precision = -1;   // (the state b2p_kernel_timing replays)
    DBuf<double> dr, dc, tmp_m, tmp_n, pv, pu, pw;
    DBuf<double> sv64, stv64;      // scaled A and A^T, FP64 (KKT, power iteration, FP64 engine)
    DBuf<float> sv32, stv32;       // scaled A and A^T, FP32 (FP32 engine)
    DBuf<double> c64, b64, l64, u64;
    DBuf<float> c32, b32, l32, u32, ylb32;  // the same in FP32 (mixed engine)
    DBuf<double> x, xa, xt, y, ya, yt;  // iterates, sized for FP64; the mixed engine stores FP32 in them
    DBuf<double> xd, yd;                 // T(z) - z of the last check (infeasibility certificates)
    bool rays = false;                   // certificates on for the current solve
    DBuf<double> xh64;                   // gathered operand, FP64 engine
    DBuf<float> xh32;                    // gathered operand of A xh, mixed engine
    // FP64 re-centring: current centre in the original space, A xbar, A^T ybar, shifted dual bound
    bool recenter = false;
    DBuf<double> xbar, ybar, axbar, atybar, ylb_s;
    DBuf<Ctrl> ctrl;
    // autotuned launch shape (lanes per row L, rows per lane group R) of the two
    // iteration kernels, keyed by the LP's shape and precision
    long long tuned_key = -1;
    int Lc = 8, Rc = 1, Lr = 8, Rr = 1, Tc = 256, Tr = 256;
    Ctrl* host_ctrl = nullptr;     // pinned, 2 slots
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~HalpernWork() {
        if (host_ctrl) cudaFreeHost(host_ctrl);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

void halpern_free(Ctx* ctx) {
    delete ctx->hw;
    ctx->hw = nullptr;
}

namespace {

constexpr int TB = 256;

__device__ __forceinline__ double block_sum_to(double v, double* slot) {
    __shared__ double sh[32];  // one slot per warp of a CTA of up to 1024 threads
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
        if (t != 0.0) atomicAdd(slot, t);
    }
    __syncthreads();
    return v;
}

template <typename T>
__device__ __forceinline__ T clampT(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------------ scaling (FP64, setup)
__global__ void k_fill(int64_t n, double v, double* __restrict__ a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v;
}

// mode 0: max |a_ij| dr_i dc_j over the segment; mode 1: sum
__global__ void k_seg_absreduce(int rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                const double* __restrict__ v, const double* __restrict__ s_self,
                                const double* __restrict__ s_other, int mode, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double acc = 0.0, si = s_self[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
            double a = fabs(v[k]) * si * s_other[idx[k]];
            acc = mode == 0 ? fmax(acc, a) : acc + a;
        }
        out[i] = acc;
    }
}

__global__ void k_div_sqrt(int64_t n, const double* __restrict__ r, double* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (r[i] > 0.0) d[i] /= sqrt(r[i]);
}

// scaled values of one CSR orientation: v_s[k] = v[k] * s_self[row] * s_other[idx[k]]
__global__ void k_scale_vals(int rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                             const double* __restrict__ v, const double* __restrict__ s_self,
                             const double* __restrict__ s_other, double* __restrict__ v64, float* __restrict__ v32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        double si = s_self[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
            double a = v[k] * si * s_other[idx[k]];
            v64[k] = a;
            if (v32) v32[k] = (float)a;
        }
    }
}

// c_s = c*dc, l_s = l/dc, u_s = u/dc ; b_s = b*dr
__global__ void k_scale_vecs(int m, int n, const double* __restrict__ b, const double* __restrict__ c,
                             const double* __restrict__ lb, const double* __restrict__ ub,
                             const double* __restrict__ dr, const double* __restrict__ dc, double* b64, double* c64,
                             double* l64, double* u64, float* b32, float* c32, float* l32, float* u32) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += st) {
        double cs = c[j] * dc[j], ls = lb[j] / dc[j], us = ub[j] / dc[j];
        c64[j] = cs; l64[j] = ls; u64[j] = us;
        if (c32) { c32[j] = (float)cs; l32[j] = (float)ls; u32[j] = (float)us; }
    }
    for (int i = tid; i < m; i += st) {
        double bs = b[i] * dr[i];
        b64[i] = bs;
        if (b32) b32[i] = (float)bs;
    }
}

// ------------------------------------------------------------------ power iteration (FP64)
// u = A_s v / nv ; v is normalised by the norm stored in *nv (1 on the first pass).
__global__ void k_pow_rows(int m, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ v64, const double* __restrict__ v, const double* __restrict__ nv,
                           double* __restrict__ u) {
    double inv = 1.0 / *nv;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) s += v64[k] * v[idx[k]];
        u[i] = s * inv;
    }
}

__global__ void k_pow_cols(int n, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const double* __restrict__ v64, const double* __restrict__ u, double* __restrict__ w,
                           double* __restrict__ nrm2) {
    double part = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; ++k) s += v64[k] * u[idx[k]];
        w[j] = s;
        part += s * s;
    }
    block_sum_to(part, nrm2);
}

__global__ void k_pow_finish(double* __restrict__ nrm2, double* __restrict__ nv, double* __restrict__ hist, int t) {
    double nn = sqrt(*nrm2);
    hist[t] = nn;          // ||A^T A v|| with ||v|| = 1  ->  sigma_max^2
    *nv = nn > 0 ? nn : 1.0;
    *nrm2 = 0.0;
}

__global__ void k_pow_init(int n, double* __restrict__ v) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        // deterministic pseudo-random start (splitmix64), entries in (0.5, 1.5)
        unsigned long long z = (unsigned long long)j * 0x9E3779B97F4A7C15ull + 0x1234567ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        v[j] = 0.5 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
    }
}

// ------------------------------------------------------------------ iterate init
// x, xa, xt <- clamp(x0 / dc) ; y, ya, yt <- P_Y(y0 / dr) (warm start given in original space;
// ZT: the iterates' storage type)
template <typename ZT>
__global__ void k_init_iterates(int m, int n, const double* __restrict__ l, const double* __restrict__ u,
                                const double* __restrict__ x0, const double* __restrict__ y0,
                                const double* __restrict__ dr, const double* __restrict__ dc,
                                const uint8_t* __restrict__ is_eq, const double* __restrict__ ylb, ZT* x, ZT* xa,
                                ZT* xt, ZT* y, ZT* ya, ZT* yt) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += st) {
        double v = x0 ? x0[j] / dc[j] : 0.0;
        v = clampT(v, l[j], u[j]);
        x[j] = (ZT)v; xa[j] = (ZT)v; xt[j] = (ZT)v;
    }
    for (int i = tid; i < m; i += st) {
        double v = y0 ? y0[i] / dr[i] : 0.0;
        const double lbv = ylb ? ylb[i] : 0.0;
        if (!is_eq[i] && v < lbv) v = lbv;
        y[i] = (ZT)v; ya[i] = (ZT)v; yt[i] = (ZT)v;
    }
}

// ------------------------------------------------------------------ iteration kernels
enum { M_PLAIN = 0, M_FIRST = 1, M_CHECK = 2 };

// VT: the iteration's type (float: mixed, double: FP64) -- matrix values, iterates,
// problem vectors, sums and updates.  GT: type of the gathered operand (y for the
// primal kernel, xh for the dual kernel), VT in both engines.
template <typename VT, typename GT>
struct IterArgs {
    const int32_t* ptr;    // CSR of the operator this kernel applies (A^T for primal, A for dual)
    const int32_t* idx;
    const VT* val;
    const GT* gather;      // y for the primal kernel, xh for the dual kernel
    const VT* cost;        // c (primal) / b (dual)
    const VT* lo;          // l (primal)
    const VT* hi;          // u (primal)
    const uint8_t* is_eq;  // dual
    const VT* ylb;         // dual: lower bound of y on <= rows in scaled space (null = 0; refinement shifts it)
    VT* z;                 // x or y, updated in place
    VT* zh;                // primal: xh out (dual: unused)
    const VT* za;          // anchor
    VT* zt;                // T(z) at check iterations
    double* zd;            // T(z) - z at check iterations (null = certificates off); dual: >= 0 on <= rows
    Ctrl* ctrl;
    int rows;
    double rho;
    const int64_t* soff;   // SELL kernel: slice offsets (ptr / idx / val unused by it except idx, val)
    const int32_t* win_lo;   // SELL kernel with gather windows: per-CTA window of `gather`
    const int32_t* win_len;  //   staged in shared memory (len 0 = none)
};

// Matrix entries and row pointers are read once per iteration: bypass L1 and mark
// them evict-first in L2, so the iterate vectors (re-read every iteration) stay
// L2-resident while the matrix streams from HBM.
__device__ __forceinline__ unsigned long long evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_stream(const float* p, unsigned long long pol) {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_stream(const double* p, unsigned long long pol) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_stream(const int* p, unsigned long long pol) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ long long ld_stream(const long long* p, unsigned long long pol) {
    long long v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
    return v;
}

// W consecutive elements (W * sizeof(T) aligned) in one or two vector loads, streaming policy.
template <int W>
__device__ __forceinline__ void ld_stream_w(const float* p, float (&v)[W], unsigned long long pol) {
    if constexpr (W == 4) {
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                     : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p), "l"(pol));
    } else if constexpr (W == 2) {
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;"
                     : "=f"(v[0]), "=f"(v[1]) : "l"(p), "l"(pol));
    } else {
        v[0] = ld_stream(p, pol);
    }
}
template <int W>
__device__ __forceinline__ void ld_stream_w(const double* p, double (&v)[W], unsigned long long pol) {
    if constexpr (W >= 2) {
#pragma unroll
        for (int h = 0; h < W; h += 2)
            asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
                         : "=d"(v[h]), "=d"(v[h + 1]) : "l"(p + h), "l"(pol));
    } else {
        v[0] = ld_stream(p, pol);
    }
}
template <int W>
__device__ __forceinline__ void ld_stream_w(const int* p, int (&v)[W], unsigned long long pol) {
    if constexpr (W == 4) {
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "l"(p), "l"(pol));
    } else if constexpr (W == 2) {
        asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.s32 {%0,%1}, [%2], %3;"
                     : "=r"(v[0]), "=r"(v[1]) : "l"(p), "l"(pol));
    } else {
        v[0] = ld_stream(p, pol);
    }
}

// Bulk prefetch of a byte range into L2 (no registers, no completion to wait for); the
// range must start on a 16-byte boundary and its size be a multiple of 16 bytes.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L lanes per row, R rows per lane group per step.  Within a step every load that
// does not depend on another -- the R row-pointer pairs, the R epilogue operands,
// the first L entries of the R rows, then their R gathers -- is issued before any
// is consumed, so each warp keeps several independent memory requests in flight
// (the kernel is bound by memory latency x parallelism, not by arithmetic).
// Each CTA owns one contiguous range of rows, so its warps gather from the same
// neighbourhood of the operand vector (for structured LPs such as block-angular
// ones, one block's slice stays in L1); the CTA size is part of the tuned shape.
// All 32 lanes of a warp stay converged through the shuffles.  Sums and updates
// are in VT; the restart residuals accumulate in FP64.
template <typename VT, typename GT, int L, int R, int MODE, bool PRIMAL>
__global__ void __launch_bounds__(1024) k_iter(IterArgs<VT, GT> a, int it) {
    const Ctrl* ctrl = a.ctrl;
    if (ctrl->done) return;
    const unsigned long long pol = evict_first_policy();
    const double kk = (double)(ctrl->k_base + it);
    const VT wk = (VT)((kk + 1.0) / (kk + 2.0));
    const VT wa = (VT)(1.0 / (kk + 2.0));
    const VT step = (VT)(PRIMAL ? ctrl->tau : ctrl->sigma);
    const VT rho = (VT)a.rho;
    const int lane = threadIdx.x & 31;
    const int sub = lane & (L - 1);
    const int rpw = 32 / L;
    const int span = rpw * R;
    const int wpc = blockDim.x >> 5;
    const int warp_in_cta = threadIdx.x >> 5;
    // this CTA's rows: [row0, row1), a multiple of span per CTA
    const long long per_cta = (((long long)a.rows + gridDim.x - 1) / gridDim.x + span - 1) / span * span;
    const int row0 = (int)min((long long)a.rows, (long long)blockIdx.x * per_cta);
    const int row1 = (int)min((long long)a.rows, (long long)row0 + per_cta);
    double acc_r = 0.0, acc_d = 0.0;
    for (int base = row0 + warp_in_cta * span; base < row1; base += wpc * span) {
        int r[R], k0[R], k1[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            r[u] = base + u * rpw + lane / L;
            const bool v = r[u] < row1;
            k0[u] = v ? ld_stream(a.ptr + r[u], pol) : 0;
            k1[u] = v ? ld_stream(a.ptr + r[u] + 1, pol) : 0;
        }
        // the row's own vectors, prefetched with the row pointers (they are only needed
        // after the reduction, so their latency overlaps the matrix stream)
        VT zr[R], cst[R], lo[R], hi[R], zan[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const bool lead = sub == 0 && r[u] < row1;
            zr[u] = lead ? a.z[r[u]] : (VT)0;
            cst[u] = lead ? a.cost[r[u]] : (VT)0;
            zan[u] = lead ? a.za[r[u]] : (VT)0;
            if (PRIMAL) {
                lo[u] = lead ? a.lo[r[u]] : (VT)0;
                hi[u] = lead ? a.hi[r[u]] : (VT)0;
            } else {
                lo[u] = (lead && !a.is_eq[r[u]]) ? (a.ylb ? a.ylb[r[u]] : (VT)0) : (VT)(-INFINITY);
                hi[u] = (VT)0;
            }
        }
        // the first two entries of every lane, all loads in flight together
        VT v[R][2];
        int c[R][2];
#pragma unroll
        for (int u = 0; u < R; ++u)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int k = k0[u] + sub + e * L;
                const bool h = k < k1[u];
                v[u][e] = h ? ld_stream(a.val + k, pol) : (VT)0;
                c[u][e] = h ? ld_stream(a.idx + k, pol) : -1;
            }
        VT s[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            s[u] = (c[u][0] >= 0) ? v[u][0] * (VT)a.gather[c[u][0]] : (VT)0;
            if (c[u][1] >= 0) s[u] += v[u][1] * (VT)a.gather[c[u][1]];
        }
#pragma unroll
        for (int u = 0; u < R; ++u)
            for (int k = k0[u] + sub + 2 * L; k < k1[u]; k += L)
                s[u] += ld_stream(a.val + k, pol) * (VT)a.gather[ld_stream(a.idx + k, pol)];
#pragma unroll
        for (int u = 0; u < R; ++u) {
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
        }
#pragma unroll
        for (int u = 0; u < R; ++u) {
            if (sub != 0 || r[u] >= row1) continue;
            const int row = r[u];
            VT zt;
            if (PRIMAL) {
                zt = clampT(zr[u] - step * (cst[u] + s[u]), lo[u], hi[u]);
                a.zh[row] = (VT)2 * zt - zr[u];
            } else {
                zt = zr[u] + step * (s[u] - cst[u]);
                if (zt < lo[u]) zt = lo[u];  // -inf on equality rows; NaN stays NaN
            }
            const VT za = zan[u];
            a.z[row] = wk * (((VT)1 + rho) * zt - rho * zr[u]) + wa * za;
            if (MODE != M_PLAIN) {
                const double d = (double)zr[u] - (double)zt;
                acc_r += d * d;
            }
            if (MODE == M_CHECK) {
                a.zt[row] = zt;
                const double dz = (double)zt - (double)zr[u];
                if (a.zd) a.zd[row] = (!PRIMAL && lo[u] != (VT)(-INFINITY)) ? fmax(dz, 0.0) : dz;
                const double e = (double)zt - (double)za;
                acc_d += e * e;
            }
        }
    }
    if (MODE == M_FIRST) block_sum_to(acc_r, &a.ctrl->acc[PRIMAL ? A_RX2_FIRST : A_RY2_FIRST]);
    if (MODE == M_CHECK) {
        block_sum_to(acc_r, &a.ctrl->acc[PRIMAL ? A_RX2 : A_RY2]);
        block_sum_to(acc_d, &a.ctrl->acc[PRIMAL ? A_DXA2 : A_DYA2]);
    }
}

// The same iteration over the SELL-32 copy: one warp per slice, one lane per row,
// so there are no row pointers to load and no shuffles, every lane of a slice runs
// the same number of chunks, and each chunk is one vector load of W values and one
// of W indices per lane (the warp reads 32 W contiguous elements of each).  Two
// chunks are loaded before either is consumed.  The row's own vectors are read
// with the slice offsets, coalesced (internal numbering).  Each CTA owns a
// contiguous range of slices.  Sums and updates in VT.
// WIN: the CTA first copies its window of the gathered vector (k_win_setup) into
// shared memory and serves the gathers that fall inside it from there -- a random
// 32-lane gather costs a few shared-memory bank cycles instead of 32 L1 requests.
// C < 32: slices of C rows, 32 / C lanes per row; the lanes of a row take every
// (32 / C)-th chunk, so one warp-wide load still reads 32 W contiguous elements, and
// their partial sums meet in a shuffle.  Smaller slices give a warp shorter chains
// and more, finer work units (better balance when there are few slices per warp).
template <typename VT, typename GT, int W, int C, int MODE, bool PRIMAL, bool WIN>
__global__ void __launch_bounds__(1024) k_iter_sell(IterArgs<VT, GT> a, int it) {
    static_assert(C == 32 || C == 16 || C == 8, "slice height");
    constexpr int LPR = 32 / C;
    const Ctrl* ctrl = a.ctrl;
    if (ctrl->done) return;
    extern __shared__ __align__(16) unsigned char win_raw[];
    GT* gwin = reinterpret_cast<GT*>(win_raw);
    int wlo = 0;
    unsigned wlen = 0;
    if (WIN) {
        wlo = a.win_lo[blockIdx.x];
        wlen = (unsigned)a.win_len[blockIdx.x];
        // 16-byte copies, 8 in flight per thread (the window starts 16-byte aligned:
        // wlo is a multiple of 4 elements), then the scalar tail
        constexpr unsigned per16 = 16 / sizeof(GT);
        const unsigned nvec = wlen / per16;
        const float4* src = reinterpret_cast<const float4*>(a.gather + wlo);
        float4* dst = reinterpret_cast<float4*>(gwin);
        for (unsigned base = threadIdx.x; base < nvec; base += 8 * blockDim.x) {
            float4 t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const unsigned j = base + u * blockDim.x;
                if (j < nvec) t[u] = src[j];
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const unsigned j = base + u * blockDim.x;
                if (j < nvec) dst[j] = t[u];
            }
        }
        for (unsigned j = nvec * per16 + threadIdx.x; j < wlen; j += blockDim.x) gwin[j] = a.gather[wlo + j];
        __syncthreads();
    }
    auto gat = [&](int c) -> GT {
        if (WIN) {
            const unsigned o = (unsigned)(c - wlo);
            return o < wlen ? gwin[o] : a.gather[c];
        }
        return a.gather[c];
    };
    const unsigned long long pol = evict_first_policy();
    const double kk = (double)(ctrl->k_base + it);
    const VT wk = (VT)((kk + 1.0) / (kk + 2.0));
    const VT wa = (VT)(1.0 / (kk + 2.0));
    const VT step = (VT)(PRIMAL ? ctrl->tau : ctrl->sigma);
    const VT rho = (VT)a.rho;
    const int lane = threadIdx.x & 31;
    const int rl = lane % C, sub = lane / C;  // row within the slice, lane group of the row
    const int wpc = blockDim.x >> 5;
    const int nsl = (a.rows + C - 1) / C;
    const int per_cta = (nsl + (int)gridDim.x - 1) / (int)gridDim.x;
    const int s0 = min(nsl, (int)blockIdx.x * per_cta);
    const int s1 = min(nsl, s0 + per_cta);
    double acc_r = 0.0, acc_d = 0.0;
    for (int sl = s0 + (threadIdx.x >> 5); sl < s1; sl += wpc) {
        const int row = sl * C + rl;
        const bool valid = row < a.rows;
        const bool lead = valid && sub == 0;
        const long long p0 = ld_stream((const long long*)a.soff + sl, pol);
        const long long p1 = ld_stream((const long long*)a.soff + sl + 1, pol);
        // the warp's next slice goes to L2 while this one is summed: its value and index
        // loads then wait on L2, not on DRAM (slice offsets are multiples of C W entries,
        // so both ranges start and end on 16-byte boundaries)
        if (lane == 0 && sl + wpc < s1) {
            const long long q0 = ld_stream((const long long*)a.soff + sl + wpc, pol);
            const long long q1 = ld_stream((const long long*)a.soff + sl + wpc + 1, pol);
            if (q1 > q0) {
                prefetch_l2(a.val + q0, (unsigned)((q1 - q0) * sizeof(VT)));
                prefetch_l2(a.idx + q0, (unsigned)((q1 - q0) * sizeof(int)));
            }
        }
        const VT zr = lead ? a.z[row] : (VT)0;
        const VT cst = lead ? a.cost[row] : (VT)0;
        const VT zan = lead ? a.za[row] : (VT)0;
        VT lo, hi = (VT)0;
        if (PRIMAL) {
            lo = lead ? a.lo[row] : (VT)0;
            hi = lead ? a.hi[row] : (VT)0;
        } else {
            lo = (lead && !a.is_eq[row]) ? (a.ylb ? a.ylb[row] : (VT)0) : (VT)(-INFINITY);
        }
        const int nq = (int)((p1 - p0) / (C * W));
        const VT* vp = a.val + p0 + rl * W;
        const int* ip = a.idx + p0 + rl * W;
        VT s_0 = (VT)0, s_1 = (VT)0;
        // chunk q of this row at vp + q C W; lane group `sub` takes q = sub, sub + LPR, ...
        // U chunks (8 entries per lane) per step: every value and index load of the step
        // (the last step predicated on the row's length) is issued before the first
        // gather, and every gather before the first multiply, so a step costs two
        // dependent L2 round trips for 8 entries
        constexpr int U = W >= 8 ? 1 : 8 / W;
        for (int q = sub; q < nq; q += U * LPR) {
            VT v[U][W];
            int c[U][W];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int qq = q + u * LPR;
                if (qq < nq) {
                    ld_stream_w<W>(vp + (int64_t)qq * C * W, v[u], pol);
                    ld_stream_w<W>(ip + (int64_t)qq * C * W, c[u], pol);
                } else {
#pragma unroll
                    for (int e = 0; e < W; ++e) {
                        v[u][e] = (VT)0;
                        c[u][e] = -1;
                    }
                }
            }
            GT g[U][W];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < W; ++e) g[u][e] = c[u][e] >= 0 ? gat(c[u][e]) : (GT)0;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    if (u & 1) s_1 += v[u][e] * (VT)g[u][e];
                    else s_0 += v[u][e] * (VT)g[u][e];
                }
        }
        VT s = s_0 + s_1;
#pragma unroll
        for (int o = C; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (!lead) continue;
        VT zt;
        if (PRIMAL) {
            zt = clampT(zr - step * (cst + s), lo, hi);
            a.zh[row] = (VT)2 * zt - zr;
        } else {
            zt = zr + step * (s - cst);
            if (zt < lo) zt = lo;  // -inf on equality rows; NaN stays NaN
        }
        a.z[row] = wk * (((VT)1 + rho) * zt - rho * zr) + wa * zan;
        if (MODE != M_PLAIN) {
            const double d = (double)zr - (double)zt;
            acc_r += d * d;
        }
        if (MODE == M_CHECK) {
            a.zt[row] = zt;
            const double dz = (double)zt - (double)zr;
            if (a.zd) a.zd[row] = (!PRIMAL && lo != (VT)(-INFINITY)) ? fmax(dz, 0.0) : dz;
            const double e = (double)zt - (double)zan;
            acc_d += e * e;
        }
    }
    if (MODE == M_FIRST) block_sum_to(acc_r, &a.ctrl->acc[PRIMAL ? A_RX2_FIRST : A_RY2_FIRST]);
    if (MODE == M_CHECK) {
        block_sum_to(acc_r, &a.ctrl->acc[PRIMAL ? A_RX2 : A_RY2]);
        block_sum_to(acc_d, &a.ctrl->acc[PRIMAL ? A_DXA2 : A_DYA2]);
    }
}

// ------------------------------------------------------------------ internal numbering and SELL copies (setup)
// key of row i: (window, decreasing length) -> a stable radix sort orders each window by length
__global__ void k_len_keys(int rows, const int32_t* __restrict__ ptr, int wlog, unsigned long long* __restrict__ keys,
                           int32_t* __restrict__ ids) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const unsigned len = (unsigned)(ptr[i + 1] - ptr[i]);
        keys[i] = ((unsigned long long)(i >> wlog) << 32) | (unsigned long long)(0xFFFFFFFFu - len);
        ids[i] = i;
    }
}

__global__ void k_invert(int rows, const int32_t* __restrict__ perm, int32_t* __restrict__ inv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) inv[perm[i]] = i;
}

// out[i + 1] = length of original row perm[i] (out[0] = 0; scanned afterwards)
__global__ void k_perm_lens(int rows, const int32_t* __restrict__ perm, const int32_t* __restrict__ ptr,
                            int32_t* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const int r = perm[i];
        out[i + 1] = ptr[r + 1] - ptr[r];
        if (i == 0) out[0] = 0;
    }
}

// internal row i = original row perm[i], its indices renumbered by imap
__global__ void k_perm_csr(int rows, const int32_t* __restrict__ perm, const int32_t* __restrict__ ptr,
                           const int32_t* __restrict__ idx, const double* __restrict__ val,
                           const int32_t* __restrict__ imap, const int32_t* __restrict__ optr,
                           int32_t* __restrict__ oidx, double* __restrict__ oval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const int r = perm[i];
        const int k0 = ptr[r], len = ptr[r + 1] - k0, o = optr[i];
        for (int e = 0; e < len; ++e) {
            oidx[o + e] = imap[idx[k0 + e]];
            oval[o + e] = val[k0 + e];
        }
    }
}

template <typename T>
__global__ void k_gather_perm(int rows, const int32_t* __restrict__ perm, const T* __restrict__ src, T* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) dst[i] = src[perm[i]];
}

template <typename T>
__global__ void k_scatter_perm(int rows, const int32_t* __restrict__ perm, const T* __restrict__ src, T* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) dst[perm[i]] = src[i];
}

// longest row of every C-row slice
__global__ void k_slice_len(int rows, const int32_t* __restrict__ ptr, int C, int32_t* __restrict__ slen) {
    const int nsl = (rows + C - 1) / C;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsl; s += gridDim.x * blockDim.x) {
        int mx = 0;
        for (int r = s * C; r < min(rows, s * C + C); ++r) mx = max(mx, ptr[r + 1] - ptr[r]);
        slen[s] = mx;
    }
}

// SELL position of entry e of row i (slices of C rows, chunks of W per lane)
__device__ __forceinline__ int64_t sell_pos(const int64_t* off, int W, int C, int i, int e) {
    return off[i / C] + (int64_t)(e / W) * C * W + (i % C) * W + (e % W);
}

// indices of the SELL copy; a padding slot repeats an index of its own row (or of the
// slice's first, longest row), so padding stays inside the row's neighbourhood of the
// gathered vector (its value is 0)
__global__ void k_sell_idx(int rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                           const int64_t* __restrict__ off, int W, int C, int32_t* __restrict__ sidx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const int k0 = ptr[i], len = ptr[i + 1] - k0;
        const int s = i / C;
        const int plen = (int)((off[s + 1] - off[s]) / C);
        for (int e = 0; e < len; ++e) sidx[sell_pos(off, W, C, i, e)] = idx[k0 + e];
        if (plen > len) {
            const int first = ptr[s * C];
            const int pad = len > 0 ? idx[k0 + len - 1] : (ptr[s * C + 1] > first ? idx[first] : 0);
            for (int e = len; e < plen; ++e) sidx[sell_pos(off, W, C, i, e)] = pad;
        }
    }
}

// Gather windows: CTA b of a grid of G over `rows` rows (contiguous ranges of
// per_cta slices, as the iteration kernel assigns them) stages the part
// [lo_b, lo_b + len_b) of the gathered vector in shared memory.  The window is
// the pair of adjacent buckets (bucket = cap / 2 elements) holding most of the
// CTA's entries; len_b = 0 (no staging) when it holds less than half of them.
__global__ void k_win_setup(int rows, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                            int per_cta, int n_other, int cap, int nb, int32_t* __restrict__ wlo,
                            int32_t* __restrict__ wlen) {
    extern __shared__ int hist[];
    const int nsl = (rows + 31) >> 5;
    const int b = blockIdx.x;
    const int s0 = min(nsl, b * per_cta), s1 = min(nsl, s0 + per_cta);
    const int r0 = min(rows, s0 * 32), r1 = min(rows, s1 * 32);
    const int bucket = cap / 2;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) hist[j] = 0;
    __syncthreads();
    const int e0 = ptr[r0], e1 = ptr[r1];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) atomicAdd(&hist[idx[e] / bucket], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int best = -1, bj = 0;
        for (int j = 0; j < nb; ++j) {
            const int c = hist[j] + (j + 1 < nb ? hist[j + 1] : 0);
            if (c > best) { best = c; bj = j; }
        }
        const int total = e1 - e0;
        int lo = bj * bucket, len = min(cap, n_other - lo);
        lo &= ~3;  // 16-byte aligned start for either element size
        len = min(cap, n_other - lo);
        const bool use = total > 0 && 2 * best >= total;
        wlo[b] = use ? lo : 0;
        wlen[b] = use ? len : 0;
    }
}

template <typename VT>
__global__ void k_sell_vals(int rows, const int32_t* __restrict__ ptr, const double* __restrict__ v64,
                            const int64_t* __restrict__ off, int W, int C, VT* __restrict__ sval) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const int k0 = ptr[i], len = ptr[i + 1] - k0;
        for (int e = 0; e < len; ++e) sval[sell_pos(off, W, C, i, e)] = (VT)v64[k0 + e];
    }
}

// ------------------------------------------------------------------ FP64 KKT of T(z) on the original LP
// rows: primal residual of x = dc*xt and the b.y term of y = dr*yt
// Point of the ORIGINAL LP that the solved problem's T(z) stands for:
//   x = xbar + pscale * dc * xt,  y = ybar + dscale * dr * yt
// (xbar = ybar = null, pscale = dscale = 1 outside refinement).  A x and A^T y of
// that point use the precomputed A xbar / A^T ybar.
struct KktMap {
    const double* xbar;   // n
    const double* ybar;   // m
    const double* axbar;  // m: A xbar
    const double* atybar; // n: A^T ybar
};

// rows: primal residual, b.y, the objective-error sum |y| viol; with xd / yd (the
// displacement T(z) - z), A xd for the primal ray and the row terms of the dual ray
template <int L, typename ZT>
__global__ void __launch_bounds__(TB) k_kkt_rows(int m, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                 const double* __restrict__ v64, const ZT* __restrict__ xt,
                                                 const ZT* __restrict__ yt, const double* __restrict__ b,
                                                 const uint8_t* __restrict__ is_eq, const double* __restrict__ dr,
                                                 KktMap map, const double* __restrict__ xd,
                                                 const double* __restrict__ yd, Ctrl* ctrl) {
    if (ctrl->done) return;
    const double ps = ctrl->pscale, ds = ctrl->dscale;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), rpw = 32 / L;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const bool rays = xd != nullptr;
    double p2 = 0.0, by = 0.0, est = 0.0, prv = 0.0, drb = 0.0, drm = 0.0, ysv = 0.0;
    for (int base = warp * rpw; base < m; base += nw * rpw) {
        int r = base + lane / L;
        bool valid = r < m;
        double s = 0.0, sd = 0.0;
        if (valid)
            for (int k = ptr[r] + sub; k < ptr[r + 1]; k += L) {
                s += v64[k] * (double)xt[idx[k]];
                if (rays) sd += v64[k] * xd[idx[k]];
            }
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            sd += __shfl_xor_sync(0xffffffffu, sd, o);
        }
        if (valid && sub == 0) {
            const bool eq = is_eq[r] != 0;
            double ax = (map.axbar ? map.axbar[r] : 0.0) + ps * (s / dr[r]);
            double rp = ax - b[r];
            if (!eq) rp = fmax(rp, 0.0);
            p2 += rp * rp;
            const double yv = (map.ybar ? map.ybar[r] : 0.0) + ds * (dr[r] * (double)yt[r]);
            by += b[r] * yv;
            est += fabs(yv) * fabs(rp);
            if (!eq && yv < 0.0) ysv += yv * yv;  // y >= 0 on <= rows: part of the dual residual
            if (rays) {
                const double adx = sd / dr[r];  // (A dx)_r, original space
                const double v = eq ? adx : fmax(adx, 0.0);
                prv += v * v;
                const double dyo = dr[r] * yd[r];
                drb += b[r] * dyo;
                drm += fabs(b[r] * dyo);
            }
        }
    }
    block_sum_to(p2, &ctrl->acc[A_PRES2]);
    block_sum_to(by, &ctrl->acc[A_BY]);
    block_sum_to(est, &ctrl->acc[A_EST]);
    block_sum_to(ysv, &ctrl->acc[A_DRES2]);
    if (rays) {
        block_sum_to(prv, &ctrl->acc[A_PRV2]);
        block_sum_to(drb, &ctrl->acc[A_DRB]);
        block_sum_to(drm, &ctrl->acc[A_DRM]);
    }
}

// columns: reduced cost g = c + A^T y, bound multipliers lambda, dual residual, c.x and the bound terms
// columns: reduced cost g = c + A^T y, bound multipliers lambda, dual residual, c.x and the bound
// terms; with xd / yd, the column terms of the primal ray and A^T yd for the dual ray
template <int L, typename ZT>
__global__ void __launch_bounds__(TB) k_kkt_cols(int n, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                                 const double* __restrict__ v64, const ZT* __restrict__ yt,
                                                 const ZT* __restrict__ xt, const double* __restrict__ c,
                                                 const double* __restrict__ lb, const double* __restrict__ ub,
                                                 const double* __restrict__ dc, KktMap map,
                                                 const double* __restrict__ xd, const double* __restrict__ yd,
                                                 Ctrl* ctrl) {
    if (ctrl->done) return;
    const double ps = ctrl->pscale, ds = ctrl->dscale;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1), rpw = 32 / L;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const bool rays = yd != nullptr;
    double d2 = 0.0, pc = 0.0, lam_t = 0.0, prv = 0.0, prc = 0.0, prm = 0.0, drl = 0.0, drm = 0.0, drv = 0.0;
    for (int base = warp * rpw; base < n; base += nw * rpw) {
        int j = base + lane / L;
        bool valid = j < n;
        double s = 0.0, sd = 0.0;
        if (valid)
            for (int k = ptr[j] + sub; k < ptr[j + 1]; k += L) {
                s += v64[k] * (double)yt[idx[k]];
                if (rays) sd += v64[k] * yd[idx[k]];
            }
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            sd += __shfl_xor_sync(0xffffffffu, sd, o);
        }
        if (valid && sub == 0) {
            double g = c[j] + (map.atybar ? map.atybar[j] : 0.0) + ds * (s / dc[j]);
            bool fl = isfinite(lb[j]), fu = isfinite(ub[j]);
            double lam = (fl && fu) ? g : (fl ? fmax(g, 0.0) : (fu ? fmin(g, 0.0) : 0.0));
            double rd = g - lam;
            d2 += rd * rd;
            double x = (map.xbar ? map.xbar[j] : 0.0) + ps * (dc[j] * (double)xt[j]);
            pc += c[j] * x;
            if (lam > 0.0) lam_t += lam * lb[j];
            else if (lam < 0.0) lam_t += lam * ub[j];
            if (rays) {
                const double dxo = dc[j] * xd[j];
                prc += c[j] * dxo;
                prm += fabs(c[j] * dxo);
                const double bv = (fl && dxo < 0.0 ? -dxo : 0.0) + (fu && dxo > 0.0 ? dxo : 0.0);
                prv += bv * bv;
                const double at = sd / dc[j];  // (A^T dy)_j, original space
                const double t = at > 0.0 ? (fl ? at * lb[j] : 0.0) : (at < 0.0 ? (fu ? at * ub[j] : 0.0) : 0.0);
                drl += t;
                drm += fabs(t);
                const double av = (!fl && at > 0.0 ? at : 0.0) + (!fu && at < 0.0 ? -at : 0.0);
                drv += av * av;
            }
        }
    }
    block_sum_to(d2, &ctrl->acc[A_DRES2]);
    block_sum_to(pc, &ctrl->acc[A_PC]);
    block_sum_to(lam_t, &ctrl->acc[A_LAM]);
    if (rays) {
        block_sum_to(prv, &ctrl->acc[A_PRV2]);
        block_sum_to(prc, &ctrl->acc[A_PRC]);
        block_sum_to(prm, &ctrl->acc[A_PRM]);
        block_sum_to(drl, &ctrl->acc[A_DRL]);
        block_sum_to(drm, &ctrl->acc[A_DRM]);
        block_sum_to(drv, &ctrl->acc[A_DRV2]);
    }
}

// One thread: termination, restart and primal-weight decisions for the chunk just run.
__global__ void k_control(Ctrl* c) {
    if (c->done) return;
    double* a = c->acc;
    double om = c->omega;
    double r = sqrt(om * a[A_RX2] + a[A_RY2] / om);
    if (c->first_after_restart) {
        c->r0 = sqrt(om * a[A_RX2_FIRST] + a[A_RY2_FIRST] / om);
        c->rprev = c->r0;
        if (c->r_first <= 0.0) c->r_first = c->r0;  // residual of the starting point of this solve
    }
    c->total += c->K;
    double pres = sqrt(a[A_PRES2]), dres = sqrt(a[A_DRES2]);
    double pobj = a[A_PC], dobj = -a[A_BY] + a[A_LAM];
    c->rel_p = pres / (1.0 + c->bnorm);
    c->rel_d = dres / (1.0 + c->cnorm);
    c->rel_g = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    c->pobj = pobj;
    c->dobj = dobj;
    c->obj_err = fmax(fmax(pobj - dobj, a[A_EST]), 0.0) / fmax(1.0, fabs(pobj));
    bool finite = isfinite(pres) && isfinite(dres) && isfinite(pobj) && isfinite(dobj) && isfinite(r);
    const bool obj_ok = c->eps_obj <= 0.0 || c->obj_err <= c->eps_obj;
    // PDLP's ratio tests on the rays; the 1e-9 floors keep the rounding noise of a
    // vanishing displacement from passing for a ray
    const bool rays = c->eps_inf > 0.0;
    const double dray = -a[A_DRB] + a[A_DRL], pray = a[A_PRC];
    const bool infeas = rays && dray > 0.0 && dray > 1e-9 * a[A_DRM] && sqrt(a[A_DRV2]) <= c->eps_inf * dray;
    const bool unbnd = rays && pray < 0.0 && -pray > 1e-9 * a[A_PRM] && sqrt(a[A_PRV2]) <= c->eps_inf * -pray;
    if (!finite) {
        c->done = 1;
        c->status = B2P_STATUS_NUMERICAL_FAILURE;
    } else if (c->rel_p <= c->eps && c->rel_d <= c->eps && c->rel_g <= c->eps && obj_ok) {
        c->done = 1;
        c->status = B2P_STATUS_OPTIMAL;
    } else if (infeas && c->inner_tol <= 0.0) {
        c->done = 1;
        c->status = B2P_STATUS_INFEASIBLE_DETECTED;
    } else if (unbnd && c->inner_tol <= 0.0) {
        c->done = 1;
        c->status = B2P_STATUS_UNBOUNDED_DETECTED;
    } else if (c->total >= c->max_iter) {
        c->done = 1;
        c->status = B2P_STATUS_MAX_ITERATIONS;
    } else if (c->inner_tol > 0.0 && r <= c->inner_tol * c->r_first) {
        c->done = 1;
        c->status = kInnerDone;
    }
    c->restart = 0;
    c->first_after_restart = 0;
    if (!c->done) {
        long long k_after = c->k_base + c->K;
        bool rs = (r <= c->beta_s * c->r0) || (r <= c->beta_n * c->r0 && r > c->rprev) ||
                  ((double)k_after >= c->beta_a * (double)c->total);
        c->rprev = r;
        if (rs) {
            double dx = sqrt(a[A_DXA2]), dy = sqrt(a[A_DYA2]);
            if (dx > 1e-10 && dy > 1e-10) {
                double nw = exp(0.5 * log(dy / dx) + 0.5 * log(om));
                if (isfinite(nw) && nw > 0.0) c->omega = nw;
            }
            c->tau = c->eta / c->omega;
            c->sigma = c->eta * c->omega;
            c->k_base = 0;
            c->restarts += 1;
            c->restart = 1;
            c->first_after_restart = 1;
        } else {
            c->k_base = k_after;
        }
    }
    for (int i = 0; i < A_COUNT; ++i) a[i] = 0.0;
}

// z <- z_anchor <- T(z) at a restart
template <typename ZT>
__global__ void k_restart(int m, int n, const Ctrl* __restrict__ c, ZT* x, ZT* xa, const ZT* __restrict__ xt, ZT* y,
                          ZT* ya, const ZT* __restrict__ yt) {
    if (c->done || !c->restart) return;
    int tid = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += st) { ZT v = xt[j]; x[j] = v; xa[j] = v; }
    for (int i = tid; i < m; i += st) { ZT v = yt[i]; y[i] = v; ya[i] = v; }
}

// unscale T(z) into FP64 outputs of the original LP: x = xbar + dc * xt, y = ybar + dr * yt
template <typename ZT>
__global__ void k_unscale(int m, int n, const ZT* __restrict__ xt, const ZT* __restrict__ yt,
                          const double* __restrict__ dr, const double* __restrict__ dc, const double* __restrict__ xbar,
                          const double* __restrict__ ybar, double* __restrict__ xo, double* __restrict__ yo) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += st) xo[j] = (xbar ? xbar[j] : 0.0) + dc[j] * (double)xt[j];
    for (int i = tid; i < m; i += st) yo[i] = (ybar ? ybar[i] : 0.0) + dr[i] * (double)yt[i];
}

// ------------------------------------------------------------------ FP64 re-centring (iterative refinement)
// At a restart the Halpern iterate and anchor become T(z).  With re-centring on,
// the problem is instead rewritten around that point (xbar, ybar) in the original
// space -- an exact change of variables, so PDHG proceeds unchanged:
//   b' = b - A xbar,  c' = c + A^T ybar,  l' = l - xbar,  u' = u - xbar,
//   y' >= -ybar on <= rows,   and the iterates restart at 0.
// A xbar and A^T ybar use the FP64 original matrix, so the FP32 matrix values
// and xh only ever act on the (small) correction: the residual is exact to FP64
// after every restart.  The three kernels return at once unless the control
// kernel has just decided to restart.
template <typename ZT>
__global__ void k_rc_update(int m, int n, const Ctrl* __restrict__ c, const double* __restrict__ dr,
                            const double* __restrict__ dc, double* xbar, double* ybar, ZT* x, ZT* xa, ZT* xt, ZT* y,
                            ZT* ya, ZT* yt) {
    if (c->done || !c->restart) return;
    int tid = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (int j = tid; j < n; j += st) {
        xbar[j] += dc[j] * (double)xt[j];
        x[j] = (ZT)0; xa[j] = (ZT)0; xt[j] = (ZT)0;
    }
    for (int i = tid; i < m; i += st) {
        ybar[i] += dr[i] * (double)yt[i];
        y[i] = (ZT)0; ya[i] = (ZT)0; yt[i] = (ZT)0;
    }
}

// The shifted problem in FP64 (bs, ylb_s) and, for the mixed engine, its FP32 copy.
__global__ void k_rc_rows(int m, const Ctrl* __restrict__ c, const int32_t* __restrict__ ptr,
                          const int32_t* __restrict__ idx, const double* __restrict__ vals,
                          const double* __restrict__ xbar, const double* __restrict__ ybar,
                          const double* __restrict__ b, const double* __restrict__ dr, double* axbar, double* bs,
                          double* ylb_s, float* bs32, float* ylb32) {
    if (c->done || !c->restart) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) s += vals[k] * xbar[idx[k]];
        axbar[i] = s;
        const double bi = dr[i] * (b[i] - s), li = -ybar[i] / dr[i];
        bs[i] = bi;
        ylb_s[i] = li;
        if (bs32) {
            bs32[i] = (float)bi;
            ylb32[i] = (float)li;
        }
    }
}

__global__ void k_rc_cols(int n, const Ctrl* __restrict__ c, const int32_t* __restrict__ ptr,
                          const int32_t* __restrict__ idx, const double* __restrict__ vals,
                          const double* __restrict__ xbar, const double* __restrict__ ybar,
                          const double* __restrict__ cost, const double* __restrict__ lb, const double* __restrict__ ub,
                          const double* __restrict__ dc, double* atybar, double* cs, double* ls, double* us, float* cs32,
                          float* ls32, float* us32) {
    if (c->done || !c->restart) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; ++k) s += vals[k] * ybar[idx[k]];
        atybar[j] = s;
        const double cj = dc[j] * (cost[j] + s), lj = (lb[j] - xbar[j]) / dc[j], uj = (ub[j] - xbar[j]) / dc[j];
        cs[j] = cj;
        ls[j] = lj;
        us[j] = uj;
        if (cs32) {
            cs32[j] = (float)cj;
            ls32[j] = (float)lj;
            us32[j] = (float)uj;
        }
    }
}

int pick_lanes(double mean_len, int requested) {
    if (requested == 1 || requested == 2 || requested == 4 || requested == 8 || requested == 16 || requested == 32)
        return requested;
    int L = 2;
    while (L < 32 && L < mean_len * 0.75) L <<= 1;
    return L;
}

template <typename VT, typename GT, int R, int MODE, bool PRIMAL>
void launch_iter_LR(int L, unsigned grid, int tb, cudaStream_t s, const IterArgs<VT, GT>& a, int it) {
    switch (L) {
        case 2: k_iter<VT, GT, 2, R, MODE, PRIMAL><<<grid, tb, 0, s>>>(a, it); break;
        case 4: k_iter<VT, GT, 4, R, MODE, PRIMAL><<<grid, tb, 0, s>>>(a, it); break;
        case 8: k_iter<VT, GT, 8, R, MODE, PRIMAL><<<grid, tb, 0, s>>>(a, it); break;
        case 16: k_iter<VT, GT, 16, R, MODE, PRIMAL><<<grid, tb, 0, s>>>(a, it); break;
        default: k_iter<VT, GT, 32, R, MODE, PRIMAL><<<grid, tb, 0, s>>>(a, it); break;
    }
}

// Plain iterations use R rows per lane group; the two reduction iterations of a chunk use R = 1.
template <typename VT, typename GT, bool PRIMAL>
void launch_iter(int mode, int L, int R, unsigned grid, int tb, cudaStream_t s, const IterArgs<VT, GT>& a, int it) {
    if (mode == M_FIRST) launch_iter_LR<VT, GT, 1, M_FIRST, PRIMAL>(L, grid, tb, s, a, it);
    else if (mode == M_CHECK) launch_iter_LR<VT, GT, 1, M_CHECK, PRIMAL>(L, grid, tb, s, a, it);
    else if (R >= 4) launch_iter_LR<VT, GT, 4, M_PLAIN, PRIMAL>(L, grid, tb, s, a, it);
    else if (R == 2) launch_iter_LR<VT, GT, 2, M_PLAIN, PRIMAL>(L, grid, tb, s, a, it);
    else launch_iter_LR<VT, GT, 1, M_PLAIN, PRIMAL>(L, grid, tb, s, a, it);
}

template <typename MT>
void launch_kkt(int Lr, int Lc, unsigned gr, unsigned gc, cudaStream_t s, const DevLP& lp, HalpernWork* w,
                const KktMap& map, Ctrl* ctrl) {
    const double* xd = w->rays ? w->xd.p : nullptr;
    const double* yd = w->rays ? w->yd.p : nullptr;
    const MT* xt = (const MT*)w->xt.p;
    const MT* yt = (const MT*)w->yt.p;
#define KR(LL) k_kkt_rows<LL, MT><<<gr, TB, 0, s>>>(lp.m, lp.rowptr.p, lp.colidx.p, w->sv64.p, xt, yt, lp.b.p, lp.is_eq.p, w->dr.p, map, xd, yd, ctrl)
#define KC(LL) k_kkt_cols<LL, MT><<<gc, TB, 0, s>>>(lp.n, lp.t_rowptr.p, lp.t_colidx.p, w->stv64.p, yt, xt, lp.c.p, lp.lb.p, lp.ub.p, w->dc.p, map, xd, yd, ctrl)
    switch (Lr) { case 1: KR(1); break; case 2: KR(2); break; case 4: KR(4); break; case 8: KR(8); break; case 16: KR(16); break; default: KR(32); }
    switch (Lc) { case 1: KC(1); break; case 2: KC(2); break; case 4: KC(4); break; case 8: KC(8); break; case 16: KC(16); break; default: KC(32); }
#undef KR
#undef KC
}

// Scaling, scaled copies and ||A_s||_2 (FP64, once per uploaded LP and ruiz count).
int prepare_scaling(Ctx* ctx, HalpernWork* w, int ruiz_iters, bool need32) {
    DevLP& L = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n;
    unsigned gm = grid_for(m, TB, ctx->sm_count), gn = grid_for(n, TB, ctx->sm_count);
    k_fill<<<gm, TB, 0, s>>>(m, 1.0, w->dr.p);
    k_fill<<<gn, TB, 0, s>>>(n, 1.0, w->dc.p);
    for (int it = 0; it < ruiz_iters; ++it) {
        k_seg_absreduce<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, w->dr.p, w->dc.p, 0, w->tmp_m.p);
        k_seg_absreduce<<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p, w->dc.p, w->dr.p, 0, w->tmp_n.p);
        k_div_sqrt<<<gm, TB, 0, s>>>(m, w->tmp_m.p, w->dr.p);
        k_div_sqrt<<<gn, TB, 0, s>>>(n, w->tmp_n.p, w->dc.p);
    }
    // Pock-Chambolle, alpha = 1
    k_seg_absreduce<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, w->dr.p, w->dc.p, 1, w->tmp_m.p);
    k_seg_absreduce<<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p, w->dc.p, w->dr.p, 1, w->tmp_n.p);
    k_div_sqrt<<<gm, TB, 0, s>>>(m, w->tmp_m.p, w->dr.p);
    k_div_sqrt<<<gn, TB, 0, s>>>(n, w->tmp_n.p, w->dc.p);
    k_scale_vals<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, L.vals.p, w->dr.p, w->dc.p, w->sv64.p,
                                   need32 ? w->sv32.p : nullptr);
    k_scale_vals<<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p, w->dc.p, w->dr.p, w->stv64.p,
                                   need32 ? w->stv32.p : nullptr);
    unsigned gmn = grid_for(std::max(m, n), TB, ctx->sm_count);
    k_scale_vecs<<<gmn, TB, 0, s>>>(m, n, L.b.p, L.c.p, L.lb.p, L.ub.p, w->dr.p, w->dc.p, w->b64.p, w->c64.p, w->l64.p,
                                    w->u64.p, need32 ? w->b32.p : nullptr, need32 ? w->c32.p : nullptr,
                                    need32 ? w->l32.p : nullptr, need32 ? w->u32.p : nullptr);
    B2P_LAUNCH(ctx);
    ctx->launches += 4 * ruiz_iters + 7;
    return B2P_OK;
}

// sigma_max(A_s)^2 by power iteration on A_s^T A_s; rounds of 16 until the estimate settles.
int power_sigma2(Ctx* ctx, HalpernWork* w, double* sigma2) {
    DevLP& L = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n;
    unsigned gm = grid_for(m, TB, ctx->sm_count), gn = grid_for(n, TB, ctx->sm_count, 4);
    double* scal = w->pw.p;  // [0] ||w||^2 accumulator, [1] ||v||, [2..17] history of ||A^T A v|| / ||v||
    const int kMax = 512, kRound = 16;
    k_pow_init<<<gn, TB, 0, s>>>(n, w->pv.p);
    k_fill<<<1, 32, 0, s>>>(2, 0.0, scal);
    B2P_LAUNCH(ctx);
    // ||v|| of the start vector (once, on the host)
    {
        std::vector<double> hv(n);
        B2P_CUDA(ctx, cudaMemcpyAsync(hv.data(), w->pv.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        double nn = 0;
        for (double v : hv) nn += v * v;
        nn = std::sqrt(nn);
        B2P_CUDA(ctx, cudaMemcpyAsync(scal + 1, &nn, sizeof(double), cudaMemcpyHostToDevice, s));
    }
    double hist[kRound];
    double est = 0.0;
    for (int t = 0; t < kMax; t += kRound) {
        for (int q = 0; q < kRound; ++q) {
            k_pow_rows<<<gm, TB, 0, s>>>(m, L.rowptr.p, L.colidx.p, w->sv64.p, w->pv.p, scal + 1, w->pu.p);
            k_pow_cols<<<gn, TB, 0, s>>>(n, L.t_rowptr.p, L.t_colidx.p, w->stv64.p, w->pu.p, w->pv.p, scal);
            k_pow_finish<<<1, 1, 0, s>>>(scal, scal + 1, scal + 2, q);
        }
        B2P_LAUNCH(ctx);
        ctx->launches += 3 * kRound;
        B2P_CUDA(ctx, cudaMemcpyAsync(hist, scal + 2, sizeof(hist), cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        est = hist[kRound - 1];
        double prev = hist[kRound - 2];
        if (est > 0 && std::fabs(est - prev) <= 1e-7 * est) break;
    }
    *sigma2 = est;
    return B2P_OK;
}

// Rows (or columns) sorted by decreasing length inside windows of 2^kWindowLog
// (stable: equal lengths keep their order).  perm: internal -> original, inv: the inverse.
constexpr int kWindowLog = 12;

int sort_by_length(Ctx* ctx, int rows, const int32_t* ptr, int32_t* perm, int32_t* inv) {
    cudaStream_t s = ctx->stream;
    DBuf<unsigned long long> keys, keys_out;
    DBuf<int32_t> ids;
    B2P_CUDA(ctx, keys.reserve(rows));
    B2P_CUDA(ctx, keys_out.reserve(rows));
    B2P_CUDA(ctx, ids.reserve(rows));
    const unsigned g = grid_for(rows, TB, ctx->sm_count);
    k_len_keys<<<g, TB, 0, s>>>(rows, ptr, kWindowLog, keys.p, ids.p);
    B2P_LAUNCH(ctx);
    int end_bit = 33;
    while (end_bit < 64 && (1LL << (end_bit - 32)) <= ((rows - 1) >> kWindowLog)) ++end_bit;
    size_t tmp = 0;
    B2P_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, keys_out.p, ids.p, perm, rows, 0, end_bit, s));
    B2P_CUDA(ctx, ctx->cub_tmp.reserve(tmp));
    tmp = ctx->cub_tmp.bytes();
    B2P_CUDA(ctx, cub::DeviceRadixSort::SortPairs(ctx->cub_tmp.p, tmp, keys.p, keys_out.p, ids.p, perm, rows, 0, end_bit, s));
    k_invert<<<g, TB, 0, s>>>(rows, perm, inv);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    B2P_CUDA(ctx, cudaStreamSynchronize(s));  // temporaries are freed on return
    return B2P_OK;
}

// One orientation of the internal CSR: internal row i is original row perm[i], its
// indices renumbered through imap.
int permute_csr(Ctx* ctx, int rows, const int32_t* perm, const int32_t* ptr, const int32_t* idx, const double* val,
                const int32_t* imap, int32_t* optr, int32_t* oidx, double* oval) {
    cudaStream_t s = ctx->stream;
    const unsigned g = grid_for(rows, TB, ctx->sm_count);
    k_perm_lens<<<g, TB, 0, s>>>(rows, perm, ptr, optr);
    B2P_LAUNCH(ctx);
    size_t tmp = 0;
    B2P_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, tmp, optr + 1, optr + 1, rows, s));
    B2P_CUDA(ctx, ctx->cub_tmp.reserve(tmp));
    tmp = ctx->cub_tmp.bytes();
    B2P_CUDA(ctx, cub::DeviceScan::InclusiveSum(ctx->cub_tmp.p, tmp, optr + 1, optr + 1, rows, s));
    k_perm_csr<<<g, TB, 0, s>>>(rows, perm, ptr, idx, val, imap, optr, oidx, oval);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    return B2P_OK;
}

// The uploaded LP in internal numbering (once per upload).
int build_internal(Ctx* ctx, HalpernWork* w) {
    const DevLP& U = ctx->lp;
    DevLP& I = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = U.m, n = U.n;
    const int64_t nnz = U.nnz;
    I.m = m;
    I.n = n;
    I.nnz = nnz;
    for (auto* b : {&w->pr, &w->ir}) B2P_CUDA(ctx, b->reserve(m));
    for (auto* b : {&w->pc, &w->ic}) B2P_CUDA(ctx, b->reserve(n));
    B2P_CUDA(ctx, I.rowptr.reserve(m + 1));
    B2P_CUDA(ctx, I.t_rowptr.reserve(n + 1));
    for (auto* b : {&I.colidx, &I.t_colidx}) B2P_CUDA(ctx, b->reserve(nnz));
    for (auto* b : {&I.vals, &I.t_vals}) B2P_CUDA(ctx, b->reserve(nnz));
    B2P_CUDA(ctx, I.b.reserve(m));
    B2P_CUDA(ctx, I.is_eq.reserve(m));
    for (auto* b : {&I.c, &I.lb, &I.ub}) B2P_CUDA(ctx, b->reserve(n));
    int st = sort_by_length(ctx, m, U.rowptr.p, w->pr.p, w->ir.p);
    if (st) return st;
    st = sort_by_length(ctx, n, U.t_rowptr.p, w->pc.p, w->ic.p);
    if (st) return st;
    st = permute_csr(ctx, m, w->pr.p, U.rowptr.p, U.colidx.p, U.vals.p, w->ic.p, I.rowptr.p, I.colidx.p, I.vals.p);
    if (st) return st;
    st = permute_csr(ctx, n, w->pc.p, U.t_rowptr.p, U.t_colidx.p, U.t_vals.p, w->ir.p, I.t_rowptr.p, I.t_colidx.p,
                     I.t_vals.p);
    if (st) return st;
    const unsigned gm = grid_for(m, TB, ctx->sm_count), gn = grid_for(n, TB, ctx->sm_count);
    k_gather_perm<double><<<gm, TB, 0, s>>>(m, w->pr.p, U.b.p, I.b.p);
    k_gather_perm<uint8_t><<<gm, TB, 0, s>>>(m, w->pr.p, U.is_eq.p, I.is_eq.p);
    k_gather_perm<double><<<gn, TB, 0, s>>>(n, w->pc.p, U.c.p, I.c.p);
    k_gather_perm<double><<<gn, TB, 0, s>>>(n, w->pc.p, U.lb.p, I.lb.p);
    k_gather_perm<double><<<gn, TB, 0, s>>>(n, w->pc.p, U.ub.p, I.ub.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 5;
    I.bnorm = U.bnorm;
    I.cnorm = U.cnorm;
    I.mean_row_len = U.mean_row_len;
    I.mean_col_len = U.mean_col_len;
    I.max_row_len = U.max_row_len;
    I.max_col_len = U.max_col_len;
    for (int k = 0; k < 3; ++k) w->sr_all[k].idx_ready = w->sc_all[k].idx_ready = false;
    w->sr = &w->sr_all[0];
    w->sc = &w->sc_all[0];
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    w->ilp_gen = ctx->lp_gen;
    return B2P_OK;
}

// Slice layout and indices of a SELL copy (once per upload): vector width W = 4 or 2
// when its padding costs at most 3 % over W = 1, which pads only to each slice's
// longest row.
int build_sell_layout(Ctx* ctx, Sell& S, int rows, const int32_t* ptr, const int32_t* idx, int C) {
    cudaStream_t s = ctx->stream;
    const int nsl = (rows + C - 1) / C;
    DBuf<int32_t> slen;
    B2P_CUDA(ctx, slen.reserve(nsl));
    k_slice_len<<<grid_for(nsl, TB, ctx->sm_count), TB, 0, s>>>(rows, ptr, C, slen.p);
    B2P_LAUNCH(ctx);
    std::vector<int32_t> h(nsl);
    B2P_CUDA(ctx, cudaMemcpyAsync(h.data(), slen.p, sizeof(int32_t) * nsl, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    auto padded_total = [&](int W) {
        int64_t t = 0;
        for (int v : h) t += (int64_t)C * ((v + W - 1) / W * W);
        return t;
    };
    const int pad_pct = 3;  // padding allowed for the wider vectors, percent of the W = 1 layout
    const int64_t t1 = padded_total(1);
    int W = 1;
    if (padded_total(4) <= t1 + t1 * pad_pct / 100) W = 4;
    else if (padded_total(2) <= t1 + t1 * pad_pct / 100) W = 2;
    std::vector<int64_t> off(nsl + 1, 0);
    for (int i = 0; i < nsl; ++i) off[i + 1] = off[i] + (int64_t)C * ((h[i] + W - 1) / W * W);
    S.C = C;
    S.W = W;
    S.slices = nsl;
    S.total = off[nsl];
    B2P_CUDA(ctx, S.off.reserve(nsl + 1));
    B2P_CUDA(ctx, S.idx.reserve(std::max<int64_t>(S.total, 1)));
    B2P_CUDA(ctx, cudaMemcpyAsync(S.off.p, off.data(), sizeof(int64_t) * (nsl + 1), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemsetAsync(S.idx.p, 0, sizeof(int32_t) * std::max<int64_t>(S.total, 1), s));
    k_sell_idx<<<grid_for(rows, TB, ctx->sm_count), TB, 0, s>>>(rows, ptr, idx, S.off.p, W, C, S.idx.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    B2P_CUDA(ctx, cudaStreamSynchronize(s));  // slen is freed on return, h / off are host temporaries
    S.idx_ready = true;
    // the value copies belong to the old layout
    S.v32.release();
    S.v64.release();
    return B2P_OK;
}

// Scaled values into a SELL copy (every solve: the scaling depends on the Ruiz count).
template <typename VT>
int fill_sell_vals(Ctx* ctx, Sell& S, int rows, const int32_t* ptr, const double* v64, DBuf<VT>& out) {
    cudaStream_t s = ctx->stream;
    const bool fresh = out.p == nullptr;
    B2P_CUDA(ctx, out.reserve(std::max<int64_t>(S.total, 1)));
    if (fresh) B2P_CUDA(ctx, cudaMemsetAsync(out.p, 0, sizeof(VT) * std::max<int64_t>(S.total, 1), s));
    k_sell_vals<VT><<<grid_for(rows, TB, ctx->sm_count), TB, 0, s>>>(rows, ptr, v64, S.off.p, S.W, S.C, out.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    return B2P_OK;
}

// Gather windows of one orientation for a windowed launch of `tb` threads and `smem`
// bytes of shared memory per CTA over a one-wave grid (per_sm CTAs per SM); gsize =
// bytes per gathered element.  Leaves W.smem = 0 when the gathered vector is too long for the bucket
// histogram (more than 16384 buckets).
int build_windows(Ctx* ctx, Win& W, int rows, const int32_t* ptr, const int32_t* idx, int n_other, int tb,
                  size_t smem, size_t gsize, int per_sm) {
    cudaStream_t s = ctx->stream;
    W.smem = 0;
    // one resident wave of `per_sm` CTAs per SM (the kernel's occupancy at this shape)
    if (per_sm < 1) return B2P_OK;
    const unsigned G = (unsigned)(ctx->sm_count * per_sm);
    const int nsl = (rows + 31) / 32;
    const int per_cta = (nsl + (int)G - 1) / (int)G;
    const int cap = (int)(smem / gsize);
    const int bucket = cap / 2;
    const long long nb = ((long long)n_other + bucket - 1) / bucket;
    if (bucket < 1 || nb > 16384) return B2P_OK;
    B2P_CUDA(ctx, W.lo.reserve(G));
    B2P_CUDA(ctx, W.len.reserve(G));
    const size_t hbytes = sizeof(int) * (size_t)nb;
    if (hbytes > 48 * 1024)
        B2P_CUDA(ctx, cudaFuncSetAttribute(k_win_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hbytes));
    k_win_setup<<<G, 256, hbytes, s>>>(rows, ptr, idx, per_cta, n_other, cap, (int)nb, W.lo.p, W.len.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    W.G = G;
    W.smem = smem;
    return B2P_OK;
}

template <typename MT>
struct Ops;
template <>
struct Ops<double> {
    static const double* sv(HalpernWork* w) { return w->sv64.p; }
    static const double* stv(HalpernWork* w) { return w->stv64.p; }
    static double* xh(HalpernWork* w) { return w->xh64.p; }
    static DBuf<double>& sell(Sell& S) { return S.v64; }
    static const double* c(HalpernWork* w) { return w->c64.p; }
    static const double* l(HalpernWork* w) { return w->l64.p; }
    static const double* u(HalpernWork* w) { return w->u64.p; }
    static const double* b(HalpernWork* w) { return w->b64.p; }
    static const double* ylb(HalpernWork* w) { return w->ylb_s.p; }
};
template <>
struct Ops<float> {
    static const float* sv(HalpernWork* w) { return w->sv32.p; }
    static const float* stv(HalpernWork* w) { return w->stv32.p; }
    static float* xh(HalpernWork* w) { return w->xh32.p; }
    static DBuf<float>& sell(Sell& S) { return S.v32; }
    static const float* c(HalpernWork* w) { return w->c32.p; }
    static const float* l(HalpernWork* w) { return w->l32.p; }
    static const float* u(HalpernWork* w) { return w->u32.p; }
    static const float* b(HalpernWork* w) { return w->b32.p; }
    static const float* ylb(HalpernWork* w) { return w->ylb32.p; }
};
// the iterates in the engine's precision (the buffers are sized for FP64)
template <typename MT>
MT* zbuf(DBuf<double>& d) { return reinterpret_cast<MT*>(d.p); }

// Arguments of the primal kernel (A^T y over A^T, updates x) and of the dual kernel
// (A xh over A, updates y; with re-centring its sign bound on <= rows is the shifted
// ylb_s), over the CSR copies or (sell = true) the SELL copies.
template <typename MT>
IterArgs<MT, MT> primal_args(const DevLP& L, HalpernWork* w, const b2p_params* p, bool sell) {
    IterArgs<MT, MT> a{L.t_rowptr.p, L.t_colidx.p, Ops<MT>::stv(w), zbuf<MT>(w->y), Ops<MT>::c(w), Ops<MT>::l(w),
                       Ops<MT>::u(w), nullptr, nullptr, zbuf<MT>(w->x), Ops<MT>::xh(w), zbuf<MT>(w->xa),
                       zbuf<MT>(w->xt), w->rays ? w->xd.p : nullptr, w->ctrl.p, L.n, p->reflection, nullptr};
    if (sell) {
        a.ptr = nullptr;
        a.idx = w->sc->idx.p;
        a.val = Ops<MT>::sell(*w->sc).p;
        a.soff = w->sc->off.p;
        a.win_lo = w->wc.lo.p;
        a.win_len = w->wc.len.p;
    }
    return a;
}
template <typename MT>
IterArgs<MT, MT> dual_args(const DevLP& L, HalpernWork* w, const b2p_params* p, bool sell) {
    IterArgs<MT, MT> a{L.rowptr.p, L.colidx.p, Ops<MT>::sv(w), Ops<MT>::xh(w), Ops<MT>::b(w), nullptr, nullptr,
                       L.is_eq.p, w->recenter ? Ops<MT>::ylb(w) : nullptr, zbuf<MT>(w->y), nullptr, zbuf<MT>(w->ya),
                       zbuf<MT>(w->yt), w->rays ? w->yd.p : nullptr, w->ctrl.p, L.m, p->reflection, nullptr};
    if (sell) {
        a.ptr = nullptr;
        a.idx = w->sr->idx.p;
        a.val = Ops<MT>::sell(*w->sr).p;
        a.soff = w->sr->off.p;
        a.win_lo = w->wr.lo.p;
        a.win_len = w->wr.len.p;
    }
    return a;
}

// Largest dynamic shared memory any windowed SELL launch asks for (bytes); every
// windowed instantiation is opened up to it once per process.
constexpr int kWinSmemMax = 200 * 1024;

template <typename VT, typename GT, int W, int C, int MODE, bool PRIMAL, bool WIN>
void launch_sell_one(unsigned grid, int tb, size_t smem, cudaStream_t s, const IterArgs<VT, GT>& a, int it) {
    if (WIN) {
        static unsigned long long opened = 0;  // host-side, per instantiation: one bit per device
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 64 && !((opened >> dev) & 1ull)) {
            cudaFuncSetAttribute(k_iter_sell<VT, GT, W, C, MODE, PRIMAL, WIN>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kWinSmemMax);
            opened |= 1ull << dev;
        }
    }
    k_iter_sell<VT, GT, W, C, MODE, PRIMAL, WIN><<<grid, tb, WIN ? smem : 0, s>>>(a, it);
}

template <typename VT, typename GT, int C, int MODE, bool PRIMAL, bool WIN>
void launch_sell_W(int W, unsigned grid, int tb, size_t smem, cudaStream_t s, const IterArgs<VT, GT>& a, int it) {
    switch (W) {
        case 4: launch_sell_one<VT, GT, 4, C, MODE, PRIMAL, WIN>(grid, tb, smem, s, a, it); break;
        case 2: launch_sell_one<VT, GT, 2, C, MODE, PRIMAL, WIN>(grid, tb, smem, s, a, it); break;
        default: launch_sell_one<VT, GT, 1, C, MODE, PRIMAL, WIN>(grid, tb, smem, s, a, it); break;
    }
}

template <typename VT, typename GT, int MODE, bool PRIMAL>
void launch_sell_CW(const Sell& S, unsigned grid, int tb, size_t smem, cudaStream_t s, const IterArgs<VT, GT>& a,
                    int it) {
    if (smem > 0) {  // gather windows: 32-row slices only
        launch_sell_W<VT, GT, 32, MODE, PRIMAL, true>(S.W, grid, tb, smem, s, a, it);
        return;
    }
    switch (S.C) {
        case 8: launch_sell_W<VT, GT, 8, MODE, PRIMAL, false>(S.W, grid, tb, 0, s, a, it); break;
        case 16: launch_sell_W<VT, GT, 16, MODE, PRIMAL, false>(S.W, grid, tb, 0, s, a, it); break;
        default: launch_sell_W<VT, GT, 32, MODE, PRIMAL, false>(S.W, grid, tb, 0, s, a, it); break;
    }
}

// smem > 0: windowed variant (a.win_lo / a.win_len set for this grid; S.C == 32), else plain SELL
template <typename VT, typename GT, bool PRIMAL>
void launch_sell(int mode, const Sell& S, unsigned grid, int tb, size_t smem, cudaStream_t s,
                 const IterArgs<VT, GT>& a, int it) {
    if (mode == M_FIRST) launch_sell_CW<VT, GT, M_FIRST, PRIMAL>(S, grid, tb, smem, s, a, it);
    else if (mode == M_CHECK) launch_sell_CW<VT, GT, M_CHECK, PRIMAL>(S, grid, tb, smem, s, a, it);
    else launch_sell_CW<VT, GT, M_PLAIN, PRIMAL>(S, grid, tb, smem, s, a, it);
}

// One resident wave: 2048 / tb CTAs per SM, each owning a contiguous row range.
inline unsigned iter_grid(int64_t rows, int L, int R, int tb, int sm_count) {
    return grid_for((rows * L + R - 1) / R, tb, sm_count, 2048 / tb);
}

// Shapes of the windowed SELL kernel tried by the tuner: (CTA size, shared memory bytes).
constexpr int kWinShapes[3][2] = {{1024, 192 * 1024}, {512, 96 * 1024}, {256, 48 * 1024}};

// Resident CTAs per SM of the windowed SELL kernel for one launch shape.
template <typename VT, typename GT, bool PRIMAL>
int sell_win_per_sm(int W, int tb, size_t smem) {
    int per = 0;
    auto q = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kWinSmemMax);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, tb, smem);
    };
    if (W == 4) q(k_iter_sell<VT, GT, 4, 32, M_PLAIN, PRIMAL, true>);
    else if (W == 2) q(k_iter_sell<VT, GT, 2, 32, M_PLAIN, PRIMAL, true>);
    else q(k_iter_sell<VT, GT, 1, 32, M_PLAIN, PRIMAL, true>);
    return per;
}

// Windows of one side for shape `k` of kWinShapes (primal gathers y, dual gathers xh; both MT).
template <typename MT>
int side_windows(Ctx* ctx, HalpernWork* w, bool primal, int k) {
    const DevLP& L = w->ilp;
    const int tb = kWinShapes[k][0];
    const size_t smem = kWinShapes[k][1];
    if (primal)
        return build_windows(ctx, w->wc, L.n, L.t_rowptr.p, L.t_colidx.p, L.m, tb, smem, sizeof(MT),
                             sell_win_per_sm<MT, MT, true>(w->sc_all[0].W, tb, smem));
    return build_windows(ctx, w->wr, L.m, L.rowptr.p, L.colidx.p, L.n, tb, smem, sizeof(MT),
                         sell_win_per_sm<MT, MT, false>(w->sr_all[0].W, tb, smem));
}

// Slice heights of the SELL layouts (index k of sr_all / sc_all).
constexpr int kSliceC[3] = {32, 16, 8};

// SELL layout k of one side with the current solve's scaled values (built on first use).
template <typename MT>
int ensure_sell(Ctx* ctx, HalpernWork* w, bool primal, int k) {
    const DevLP& L = w->ilp;
    Sell& S = primal ? w->sc_all[k] : w->sr_all[k];
    if (S.idx_ready) return B2P_OK;
    int st = primal ? build_sell_layout(ctx, S, L.n, L.t_rowptr.p, L.t_colidx.p, kSliceC[k])
                    : build_sell_layout(ctx, S, L.m, L.rowptr.p, L.colidx.p, kSliceC[k]);
    if (st) return st;
    return primal ? fill_sell_vals<MT>(ctx, S, L.n, L.t_rowptr.p, w->stv64.p, Ops<MT>::sell(S))
                  : fill_sell_vals<MT>(ctx, S, L.m, L.rowptr.p, w->sv64.p, Ops<MT>::sell(S));
}

// Times candidate launch shapes of the primal and dual kernels on the uploaded LP
// (plain iterations from the current iterates, CUDA events on the context stream)
// and keeps the fastest of each side: the SELL kernel with slice heights 32 / 16 / 8
// (1 / 2 / 4 lanes per row) and CTA sizes 256 / 512 / 1024, the SELL kernel with
// gather windows in shared memory (32-row slices, kWinShapes), and the CSR kernel
// with (L lanes per row, R rows per lane group, CTA size).  The caller
// re-initialises the iterates afterwards.  lanes_per_row > 0 forces the CSR kernel
// with that L, -1 the SELL kernel (32-row slices, CTA size 256), -2 the windowed
// SELL kernel (CTA size 512, 96 KB), -3 / -4 the SELL kernel with 16- / 8-row slices
// (CTA size 256); each skips the search.
template <typename MT>
int autotune_shapes(Ctx* ctx, HalpernWork* w, const b2p_params* p) {
    DevLP& L = w->ilp;
    const long long key = ((long long)L.nnz * 1000003LL + (long long)L.m * 101LL + L.n) * 2 + (sizeof(MT) == 4);
    if (p->lanes_per_row != 0) {
        const bool sell = p->lanes_per_row < 0;
        const int k = p->lanes_per_row == -3 ? 1 : (p->lanes_per_row == -4 ? 2 : 0);
        w->sell_c = w->sell_r = sell;
        w->Lc = w->Lr = sell ? 32 / kSliceC[k] : pick_lanes(0, p->lanes_per_row);
        w->Rc = w->Rr = 1;
        w->Tc = w->Tr = 256;
        w->wc.smem = w->wr.smem = 0;
        for (int side = 0; side < 2 && sell; ++side) {
            int st = ensure_sell<MT>(ctx, w, side == 0, k);
            if (st) return st;
        }
        w->sc = &w->sc_all[k];
        w->sr = &w->sr_all[k];
        if (p->lanes_per_row == -2) {
            w->Tc = w->Tr = kWinShapes[1][0];
            for (int side = 0; side < 2; ++side) {
                int st = side_windows<MT>(ctx, w, side == 0, 1);
                if (st) return st;
            }
        }
        w->tuned_key = -1;
        return B2P_OK;
    }
    if (w->tuned_key == key) {
        // same size as the tuned LP (possibly another upload): its layouts and windows
        for (int side = 0; side < 2; ++side) {
            const bool primal = side == 0;
            const int k = primal ? w->kc_t : w->kr_t, wk = primal ? w->winc_t : w->winr_t;
            int st = ensure_sell<MT>(ctx, w, primal, k);
            if (st) return st;
            (primal ? w->sc : w->sr) = &(primal ? w->sc_all : w->sr_all)[k];
            (primal ? w->wc : w->wr).smem = 0;
            if (wk >= 0) {
                st = side_windows<MT>(ctx, w, primal, wk);
                if (st) return st;
            }
        }
        return B2P_OK;
    }
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n;
    cudaEvent_t e0, e1;
    B2P_CUDA(ctx, cudaEventCreate(&e0));
    B2P_CUDA(ctx, cudaEventCreate(&e1));
    for (int side = 0; side < 2; ++side) {
        const bool primal = side == 0;
        const int64_t rows = primal ? n : m;
        const double mean = primal ? L.mean_col_len : L.mean_row_len;
        const int base_L = pick_lanes(mean, 0);
        Win& win = primal ? w->wc : w->wr;
        Sell** cur = primal ? &w->sc : &w->sr;
        Sell* all = primal ? w->sc_all : w->sr_all;
        float best = 1e30f;
        int bestL = base_L, bestR = 1, bestT = 256, bestWin = -1, bestK = 0;
        bool bestS = false;
        // kind 0: CSR (Lc, R, tb); 1: SELL (layout k, tb); 2: windowed SELL (32-row slices, shape k)
        auto trial = [&](int kind, int Lc, int R, int tb, int k) -> int {
            unsigned g;
            size_t smem = 0;
            if (kind == 2) {
                *cur = &all[0];
                int st = side_windows<MT>(ctx, w, primal, k);
                if (st) return st;
                if (win.smem == 0) return B2P_OK;  // not possible for this LP
                g = win.G;
                smem = win.smem;
            } else if (kind == 1) {
                int st = ensure_sell<MT>(ctx, w, primal, k);
                if (st) return st;
                *cur = &all[k];
                win.smem = 0;
                g = iter_grid(rows, 32 / kSliceC[k], 1, tb, ctx->sm_count);
            } else {
                win.smem = 0;
                g = iter_grid(rows, Lc, R, tb, ctx->sm_count);
            }
            const IterArgs<MT, MT> pa = primal_args<MT>(L, w, p, kind != 0);
            const IterArgs<MT, MT> da = dual_args<MT>(L, w, p, kind != 0);
            float tot = 0.f;
            for (int rep = 0; rep < 4; ++rep) {
                cudaEventRecord(e0, s);
                if (kind != 0 && primal) launch_sell<MT, MT, true>(M_PLAIN, **cur, g, tb, smem, s, pa, rep);
                else if (kind != 0) launch_sell<MT, MT, false>(M_PLAIN, **cur, g, tb, smem, s, da, rep);
                else if (primal) launch_iter<MT, MT, true>(M_PLAIN, Lc, R, g, tb, s, pa, rep);
                else launch_iter<MT, MT, false>(M_PLAIN, Lc, R, g, tb, s, da, rep);
                cudaEventRecord(e1, s);
                B2P_LAUNCH(ctx);
                B2P_CUDA(ctx, cudaEventSynchronize(e1));
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) tot += ms;  // first launch warms caches
            }
            ctx->launches += 4;
            if (tot < best) {
                best = tot;
                bestS = kind != 0;
                bestWin = kind == 2 ? k : -1;
                bestK = kind == 1 ? k : 0;
                bestL = kind == 1 ? 32 / kSliceC[k] : Lc;
                bestR = R;
                bestT = tb;
            }
            return B2P_OK;
        };
        for (int k = 0; k < 3; ++k)
            for (int tb : {256, 512, 1024}) {
                int st = trial(1, 1, 1, tb, k);
                if (st) return st;
            }
        for (int k = 0; k < 3; ++k) {
            int st = trial(2, 1, 1, kWinShapes[k][0], k);
            if (st) return st;
        }
        for (int Lc : {base_L / 2, base_L, base_L * 2}) {
            if (Lc < 2 || Lc > 32) continue;
            for (int R : {1, 2, 4})
                for (int tb : {256, 512, 1024}) {
                    int st = trial(0, Lc, R, tb, 0);
                    if (st) return st;
                }
        }
        win.smem = 0;
        *cur = &all[bestK];
        if (bestWin >= 0) {
            int st = side_windows<MT>(ctx, w, primal, bestWin);
            if (st) return st;
        }
        if (primal) {
            w->sell_c = bestS; w->Lc = bestL; w->Rc = bestR; w->Tc = bestT;
            w->kc_t = bestK; w->winc_t = bestWin;
        } else {
            w->sell_r = bestS; w->Lr = bestL; w->Rr = bestR; w->Tr = bestT;
            w->kr_t = bestK; w->winr_t = bestWin;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    w->tuned_key = key;
    return B2P_OK;
}

template <typename MT>
int run_chunks(Ctx* ctx, HalpernWork* w, const b2p_params* p, double time_limit_ms, double t_start) {
    DevLP& L = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n, K = p->check_every;
    const bool mixed = sizeof(MT) == 4;
    const int Lr = w->Lr, Lc = w->Lc, Rr = w->Rr, Rc = w->Rc, Tr = w->Tr, Tc = w->Tc;
    // R = 1 grids serve the two reduction iterations; the KKT kernels use 256-thread grids
    unsigned gr = iter_grid(m, Lr, 1, Tr, ctx->sm_count), gc = iter_grid(n, Lc, 1, Tc, ctx->sm_count);
    unsigned grR = iter_grid(m, Lr, Rr, Tr, ctx->sm_count), gcR = iter_grid(n, Lc, Rc, Tc, ctx->sm_count);
    // SELL grids: one thread per row, or the windows' one-wave grid
    const unsigned grS = w->wr.smem ? w->wr.G : gr, gcS = w->wc.smem ? w->wc.G : gc;
    const int Lkr = pick_lanes(L.mean_row_len, 0), Lkc = pick_lanes(L.mean_col_len, 0);
    unsigned gkr = iter_grid(m, Lkr, 1, TB, ctx->sm_count), gkc = iter_grid(n, Lkc, 1, TB, ctx->sm_count);
    Ctrl* ctrl = w->ctrl.p;
    const IterArgs<MT, MT> pa = primal_args<MT>(L, w, p, w->sell_c);
    const IterArgs<MT, MT> da = dual_args<MT>(L, w, p, w->sell_r);
    auto chunk = [&]() {
        for (int i = 0; i < K; ++i) {
            int mode = (i == 0) ? M_FIRST : (i == K - 1 ? M_CHECK : M_PLAIN);
            if (w->sell_c) launch_sell<MT, MT, true>(mode, *w->sc, gcS, Tc, w->wc.smem, s, pa, i);
            else if (mode == M_PLAIN) launch_iter<MT, MT, true>(mode, Lc, Rc, gcR, Tc, s, pa, i);
            else launch_iter<MT, MT, true>(mode, Lc, 1, gc, Tc, s, pa, i);
            if (w->sell_r) launch_sell<MT, MT, false>(mode, *w->sr, grS, Tr, w->wr.smem, s, da, i);
            else if (mode == M_PLAIN) launch_iter<MT, MT, false>(mode, Lr, Rr, grR, Tr, s, da, i);
            else launch_iter<MT, MT, false>(mode, Lr, 1, gr, Tr, s, da, i);
        }
        const KktMap map = w->recenter ? KktMap{w->xbar.p, w->ybar.p, w->axbar.p, w->atybar.p}
                                       : KktMap{nullptr, nullptr, nullptr, nullptr};
        launch_kkt<MT>(Lkr, Lkc, gkr, gkc, s, L, w, map, ctrl);
        k_control<<<1, 1, 0, s>>>(ctrl);
        const unsigned gv = grid_for(std::max(m, n), TB, ctx->sm_count, 8);
        if (w->recenter) {
            k_rc_update<MT><<<gv, TB, 0, s>>>(m, n, ctrl, w->dr.p, w->dc.p, w->xbar.p, w->ybar.p, zbuf<MT>(w->x),
                                              zbuf<MT>(w->xa), zbuf<MT>(w->xt), zbuf<MT>(w->y), zbuf<MT>(w->ya),
                                              zbuf<MT>(w->yt));
            k_rc_rows<<<grid_for(m, TB, ctx->sm_count, 8), TB, 0, s>>>(m, ctrl, L.rowptr.p, L.colidx.p, L.vals.p,
                                                                      w->xbar.p, w->ybar.p, L.b.p, w->dr.p,
                                                                      w->axbar.p, w->b64.p, w->ylb_s.p,
                                                                      mixed ? w->b32.p : nullptr,
                                                                      mixed ? w->ylb32.p : nullptr);
            k_rc_cols<<<grid_for(n, TB, ctx->sm_count, 8), TB, 0, s>>>(n, ctrl, L.t_rowptr.p, L.t_colidx.p, L.t_vals.p,
                                                                      w->xbar.p, w->ybar.p, L.c.p, L.lb.p, L.ub.p,
                                                                      w->dc.p, w->atybar.p, w->c64.p, w->l64.p,
                                                                      w->u64.p, mixed ? w->c32.p : nullptr,
                                                                      mixed ? w->l32.p : nullptr,
                                                                      mixed ? w->u32.p : nullptr);
        } else {
            k_restart<MT><<<gv, TB, 0, s>>>(m, n, ctrl, zbuf<MT>(w->x), zbuf<MT>(w->xa), zbuf<MT>(w->xt),
                                            zbuf<MT>(w->y), zbuf<MT>(w->ya), zbuf<MT>(w->yt));
        }
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    B2P_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    chunk();
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) {
        ctx->err = std::string("graph capture: ") + cudaGetErrorString(ce);
        return B2P_EXECUTION_FAILED;
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        ctx->err = std::string("graph instantiate: ") + cudaGetErrorString(ce);
        return B2P_EXECUTION_FAILED;
    }
    const int64_t per_chunk = 2 * K + 4;
    int64_t launched = 0;
    int slot = 0;
    bool timed_out = false;
    // depth-2 pipeline: chunk r+1 is queued before the host waits on chunk r's control block
    B2P_CUDA(ctx, cudaGraphLaunch(exec, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(&w->host_ctrl[0], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaEventRecord(w->ev[0], s));
    launched++;
    const int64_t max_chunks = (p->max_iterations + K - 1) / K + 2;
    while (true) {
        int nxt = slot ^ 1;
        if (launched < max_chunks) {
            B2P_CUDA(ctx, cudaGraphLaunch(exec, s));
            B2P_CUDA(ctx, cudaMemcpyAsync(&w->host_ctrl[nxt], ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
            B2P_CUDA(ctx, cudaEventRecord(w->ev[nxt], s));
            launched++;
        }
        B2P_CUDA(ctx, cudaEventSynchronize(w->ev[slot]));
        if (w->host_ctrl[slot].done) break;
        if (launched >= max_chunks) {
            B2P_CUDA(ctx, cudaEventSynchronize(w->ev[nxt]));
            break;
        }
        if (time_limit_ms > 0 && now_ms() - t_start > time_limit_ms) {
            timed_out = true;
            break;
        }
        slot = nxt;
    }
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    ctx->launches += launched * per_chunk;
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    return timed_out ? B2P_TIMEOUT : B2P_OK;
}

template <typename MT>
int solve_T(Ctx* ctx, HalpernWork* w, const b2p_params* p, const double* x0, const double* y0, b2p_result* r,
            double* x_out, double* y_out) {
    DevLP& L = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n;
    const bool mixed = sizeof(MT) == 4;
    double t_start = now_ms();
    if (mixed) {
        B2P_CUDA(ctx, w->xh32.reserve(n));
        B2P_CUDA(ctx, w->sv32.reserve(L.nnz));
        B2P_CUDA(ctx, w->stv32.reserve(L.nnz));
    } else {
        B2P_CUDA(ctx, w->xh64.reserve(n));
    }
    // re-centring (FP64 iterative refinement at every restart): on by default for the
    // mixed engine, off for FP64; refinement_rounds > 0 forces it on, 0 off
    w->recenter = p->refinement_rounds > 0 || (p->refinement_rounds < 0 && mixed);
    if (w->recenter) {
        for (auto* b : {&w->xbar, &w->atybar}) {
            B2P_CUDA(ctx, b->reserve(n));
            B2P_CUDA(ctx, cudaMemsetAsync(b->p, 0, sizeof(double) * n, s));
        }
        for (auto* b : {&w->ybar, &w->axbar, &w->ylb_s}) {
            B2P_CUDA(ctx, b->reserve(m));
            B2P_CUDA(ctx, cudaMemsetAsync(b->p, 0, sizeof(double) * m, s));
        }
        if (mixed) {
            B2P_CUDA(ctx, w->ylb32.reserve(m));
            B2P_CUDA(ctx, cudaMemsetAsync(w->ylb32.p, 0, sizeof(float) * m, s));
        }
    }
    w->rays = p->eps_infeasible > 0.0;
    if (w->rays) {
        B2P_CUDA(ctx, w->xd.reserve(n));
        B2P_CUDA(ctx, w->yd.reserve(m));
    }
    int st = prepare_scaling(ctx, w, p->ruiz_iterations, mixed);
    if (st) return st;
    // SELL layouts: the 32-row one always, the others once the tuner has built them;
    // every built layout gets this solve's scaled values
    for (int k = 0; k < 3; ++k) {
        Sell& R = w->sr_all[k];
        Sell& Cc = w->sc_all[k];
        if (k == 0 && !R.idx_ready) {
            st = build_sell_layout(ctx, R, m, L.rowptr.p, L.colidx.p, kSliceC[0]);
            if (st) return st;
        }
        if (k == 0 && !Cc.idx_ready) {
            st = build_sell_layout(ctx, Cc, n, L.t_rowptr.p, L.t_colidx.p, kSliceC[0]);
            if (st) return st;
        }
        if (R.idx_ready) {
            st = fill_sell_vals<MT>(ctx, R, m, L.rowptr.p, w->sv64.p, Ops<MT>::sell(R));
            if (st) return st;
        }
        if (Cc.idx_ready) {
            st = fill_sell_vals<MT>(ctx, Cc, n, L.t_rowptr.p, w->stv64.p, Ops<MT>::sell(Cc));
            if (st) return st;
        }
    }
    double sig2 = 0.0;
    st = power_sigma2(ctx, w, &sig2);
    if (st) return st;
    double sigma_max = std::sqrt(std::max(sig2, 0.0));
    double eta = sigma_max > 0 ? p->step_safety / sigma_max : 1.0;
    double omega = p->primal_weight;
    if (!(omega > 0)) {  // ||c_s|| / ||b_s||
        std::vector<double> hb(m), hc(n);
        B2P_CUDA(ctx, cudaMemcpyAsync(hb.data(), w->b64.p, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(hc.data(), w->c64.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        double bn = 0, cn = 0;
        for (double v : hb) bn += v * v;
        for (double v : hc) cn += v * v;
        bn = std::sqrt(bn);
        cn = std::sqrt(cn);
        omega = (bn > 1e-10 && cn > 1e-10) ? cn / bn : 1.0;
    }
    // warm start (original space) -> device temporaries
    const double* x0d = nullptr;
    const double* y0d = nullptr;
    if (x0) {  // original -> internal numbering (pv / pu are free after the power iteration)
        B2P_CUDA(ctx, cudaMemcpyAsync(w->tmp_n.p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        k_gather_perm<double><<<grid_for(n, TB, ctx->sm_count), TB, 0, s>>>(n, w->pc.p, w->tmp_n.p, w->pv.p);
        B2P_LAUNCH(ctx);
        ctx->launches += 1;
        x0d = w->pv.p;
    }
    if (y0) {
        B2P_CUDA(ctx, cudaMemcpyAsync(w->tmp_m.p, y0, sizeof(double) * m, cudaMemcpyHostToDevice, s));
        k_gather_perm<double><<<grid_for(m, TB, ctx->sm_count), TB, 0, s>>>(m, w->pr.p, w->tmp_m.p, w->pu.p);
        B2P_LAUNCH(ctx);
        ctx->launches += 1;
        y0d = w->pu.p;
    }
    k_init_iterates<MT><<<grid_for(std::max(m, n), TB, ctx->sm_count), TB, 0, s>>>(
        m, n, w->l64.p, w->u64.p, x0d, y0d, w->dr.p, w->dc.p, L.is_eq.p, nullptr, zbuf<MT>(w->x), zbuf<MT>(w->xa),
        zbuf<MT>(w->xt), zbuf<MT>(w->y), zbuf<MT>(w->ya), zbuf<MT>(w->yt));
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    Ctrl hc;
    std::memset(&hc, 0, sizeof(hc));
    hc.omega = omega;
    hc.eta = eta;
    hc.tau = eta / omega;
    hc.sigma = eta * omega;
    hc.eps = p->eps_rel_kkt;
    hc.eps_obj = p->eps_objective;
    hc.eps_inf = w->rays ? p->eps_infeasible : 0.0;
    hc.beta_s = p->restart_sufficient;
    hc.beta_n = p->restart_necessary;
    hc.beta_a = p->restart_artificial;
    hc.bnorm = L.bnorm;
    hc.cnorm = L.cnorm;
    hc.max_iter = p->max_iterations;
    hc.K = p->check_every;
    hc.first_after_restart = 1;
    hc.status = B2P_STATUS_MAX_ITERATIONS;
    hc.pscale = 1.0;
    hc.dscale = 1.0;
    hc.inner_tol = 0.0;
    hc.r_first = 0.0;
    B2P_CUDA(ctx, cudaMemcpyAsync(w->ctrl.p, &hc, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
    {
        const long long before = w->tuned_key;
        st = autotune_shapes<MT>(ctx, w, p);  // returns at once when this LP shape is already tuned
        if (st) return st;
        if (before != w->tuned_key && w->tuned_key >= 0) {  // the trial iterations moved the iterates: reset
            k_init_iterates<MT><<<grid_for(std::max(m, n), TB, ctx->sm_count), TB, 0, s>>>(
                m, n, w->l64.p, w->u64.p, x0d, y0d, w->dr.p, w->dc.p, L.is_eq.p, nullptr, zbuf<MT>(w->x),
                zbuf<MT>(w->xa), zbuf<MT>(w->xt), zbuf<MT>(w->y), zbuf<MT>(w->ya), zbuf<MT>(w->yt));
            B2P_LAUNCH(ctx);
            ctx->launches += 1;
            B2P_CUDA(ctx, cudaMemcpyAsync(w->ctrl.p, &hc, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
        }
    }
    w->solved_gen = ctx->lp_gen;
    w->solved_precision = p->precision;
    B2P_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
    st = run_chunks<MT>(ctx, w, p, p->time_limit_s * 1000.0, t_start);
    B2P_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
    if (st != B2P_OK && st != B2P_TIMEOUT) return st;
    Ctrl fin;
    B2P_CUDA(ctx, cudaMemcpyAsync(&fin, w->ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    float kms = 0.f;
    cudaEventElapsedTime(&kms, ctx->ev0, ctx->ev1);
    r->kernel_time_ms = kms;
    r->status = st == B2P_TIMEOUT ? B2P_STATUS_INTERRUPTED : fin.status;
    r->iterations = fin.total;
    r->restarts = fin.restarts;
    r->primal_objective = fin.pobj;
    r->dual_objective = fin.dobj;
    r->rel_primal_residual = fin.rel_p;
    r->rel_dual_residual = fin.rel_d;
    r->rel_gap = fin.rel_g;
    r->rel_kkt = std::max(fin.rel_p, std::max(fin.rel_d, fin.rel_g));
    r->primal_weight = fin.omega;
    r->step_size = eta;
    r->refinement_rounds_done = w->recenter ? (int)fin.restarts : 0;
    if (x_out || y_out) {
        double t0 = now_ms();
        k_unscale<MT><<<grid_for(std::max(m, n), TB, ctx->sm_count), TB, 0, s>>>(
            m, n, zbuf<MT>(w->xt), zbuf<MT>(w->yt), w->dr.p, w->dc.p, w->recenter ? w->xbar.p : nullptr,
            w->recenter ? w->ybar.p : nullptr, w->tmp_n.p, w->tmp_m.p);
        // internal -> original numbering
        k_scatter_perm<double><<<grid_for(n, TB, ctx->sm_count), TB, 0, s>>>(n, w->pc.p, w->tmp_n.p, w->pv.p);
        k_scatter_perm<double><<<grid_for(m, TB, ctx->sm_count), TB, 0, s>>>(m, w->pr.p, w->tmp_m.p, w->pu.p);
        B2P_LAUNCH(ctx);
        ctx->launches += 3;
        if (x_out) B2P_CUDA(ctx, cudaMemcpyAsync(x_out, w->pv.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        if (y_out) B2P_CUDA(ctx, cudaMemcpyAsync(y_out, w->pu.p, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        r->transfer_time_ms += now_ms() - t0;
    }
    return B2P_OK;
}

template <typename MT>
int kernel_timing_T(Ctx* ctx, HalpernWork* w, const b2p_params* p, int reps, double* pms, double* dms, double* pb,
                    double* db) {
    DevLP& L = w->ilp;
    cudaStream_t s = ctx->stream;
    const int m = L.m, n = L.n;
    const int Lr = w->Lr, Lc = w->Lc, Rr = w->Rr, Rc = w->Rc, Tr = w->Tr, Tc = w->Tc;
    unsigned gr = iter_grid(m, Lr, w->sell_r ? 1 : Rr, Tr, ctx->sm_count);
    unsigned gc = iter_grid(n, Lc, w->sell_c ? 1 : Rc, Tc, ctx->sm_count);
    if (w->sell_r && w->wr.smem) gr = w->wr.G;
    if (w->sell_c && w->wc.smem) gc = w->wc.G;
    Ctrl* ctrl = w->ctrl.p;
    // re-open the (finished) control block for plain iterations, restore it afterwards
    Ctrl saved;
    B2P_CUDA(ctx, cudaMemcpyAsync(&saved, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    Ctrl open = saved;
    open.done = 0;
    B2P_CUDA(ctx, cudaMemcpyAsync(ctrl, &open, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
    const IterArgs<MT, MT> pa = primal_args<MT>(L, w, p, w->sell_c);
    const IterArgs<MT, MT> da = dual_args<MT>(L, w, p, w->sell_r);
    cudaEvent_t e[3];
    for (auto& x : e) B2P_CUDA(ctx, cudaEventCreate(&x));
    double tp = 0, td = 0;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e[0], s);
        if (w->sell_c) launch_sell<MT, MT, true>(M_PLAIN, *w->sc, gc, Tc, w->wc.smem, s, pa, r);
        else launch_iter<MT, MT, true>(M_PLAIN, Lc, Rc, gc, Tc, s, pa, r);
        cudaEventRecord(e[1], s);
        if (w->sell_r) launch_sell<MT, MT, false>(M_PLAIN, *w->sr, gr, Tr, w->wr.smem, s, da, r);
        else launch_iter<MT, MT, false>(M_PLAIN, Lr, Rr, gr, Tr, s, da, r);
        cudaEventRecord(e[2], s);
        B2P_LAUNCH(ctx);
        B2P_CUDA(ctx, cudaEventSynchronize(e[2]));
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e[0], e[1]);
        cudaEventElapsedTime(&b, e[1], e[2]);
        tp += a;
        td += b;
    }
    ctx->launches += 2LL * reps;
    for (auto& x : e) cudaEventDestroy(x);
    B2P_CUDA(ctx, cudaMemcpyAsync(ctrl, &saved, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    *pms = tp / reps;
    *dms = td / reps;
    // algorithmic bytes: every matrix entry, row pointer (CSR) or slice offset (SELL) and
    // vector element once; SELL padding is not counted
    const double vb = sizeof(MT), nnz = (double)L.nnz;
    const double pc_bytes = w->sell_c ? 8.0 * (w->sc->slices + 1) : 4.0 * (n + 1);
    const double pr_bytes = w->sell_r ? 8.0 * (w->sr->slices + 1) : 4.0 * (m + 1);
    // primal: A^T values+indices, col pointers, gather y, x r/w, xa, c, l, u, xh write (vb bytes each)
    *pb = nnz * (vb + 4) + pc_bytes + vb * m + n * (vb * 7);
    // dual: A values+indices, row pointers, gather xh, y r/w, ya, b, dual bound (vb each), is_eq (1)
    *db = nnz * (vb + 4) + pr_bytes + vb * n + m * (vb * 5 + 1);
    return B2P_OK;
}

}  // namespace

int halpern_kernel_timing(Ctx* ctx, const b2p_params* p, int reps, double* primal_ms, double* dual_ms,
                          double* primal_bytes, double* dual_bytes) {
    HalpernWork* w = ctx->hw;
    if (w->solved_gen != ctx->lp_gen || w->solved_precision != p->precision) {
        ctx->err = "b2p_kernel_timing: the last solve of the uploaded LP used another precision (or none ran)";
        return B2P_NO_LP;
    }
    if (p->precision == B2P_FP32) {
        if (!w->xh32.p || !w->sv32.p) {
            ctx->err = "b2p_kernel_timing: no mixed-precision solve to time";
            return B2P_NO_LP;
        }
        return kernel_timing_T<float>(ctx, w, p, reps, primal_ms, dual_ms, primal_bytes, dual_bytes);
    }
    if (!w->xh64.p) {
        ctx->err = "b2p_kernel_timing: no FP64 solve to time";
        return B2P_NO_LP;
    }
    return kernel_timing_T<double>(ctx, w, p, reps, primal_ms, dual_ms, primal_bytes, dual_bytes);
}

int halpern_engine_solve(Ctx* ctx, const b2p_params* p, const double* x0, const double* y0, b2p_result* r,
                         double* x_out, double* y_out) {
    if (p->check_every < 2) {
        ctx->err = "check_every must be >= 2";
        return B2P_INVALID_ARGUMENT;
    }
    if (p->precision != B2P_FP64 && p->precision != B2P_FP32) {
        ctx->err = "unknown precision";
        return B2P_INVALID_ARGUMENT;
    }
    if (!ctx->hw) ctx->hw = new HalpernWork();
    HalpernWork* w = ctx->hw;
    if (w->ilp_gen != ctx->lp_gen) {
        int st = build_internal(ctx, w);
        if (st) return st;
    }
    DevLP& L = w->ilp;
    const int m = L.m, n = L.n;
    const int64_t nnz = L.nnz;
    w->m = m;
    w->n = n;
    for (auto* b : {&w->dc, &w->tmp_n, &w->pv, &w->c64, &w->l64, &w->u64, &w->x, &w->xa, &w->xt})
        B2P_CUDA(ctx, b->reserve(n));
    for (auto* b : {&w->dr, &w->tmp_m, &w->pu, &w->b64, &w->y, &w->ya, &w->yt}) B2P_CUDA(ctx, b->reserve(m));
    if (p->precision == B2P_FP32) {
        for (auto* b : {&w->c32, &w->l32, &w->u32}) B2P_CUDA(ctx, b->reserve(n));
        for (auto* b : {&w->b32, &w->ylb32}) B2P_CUDA(ctx, b->reserve(m));
    }
    B2P_CUDA(ctx, w->pw.reserve(64));
    B2P_CUDA(ctx, w->sv64.reserve(nnz));
    B2P_CUDA(ctx, w->stv64.reserve(nnz));
    B2P_CUDA(ctx, w->ctrl.reserve(1));
    if (!w->host_ctrl) B2P_CUDA(ctx, cudaMallocHost(&w->host_ctrl, 2 * sizeof(Ctrl)));
    for (auto& e : w->ev)
        if (!e) B2P_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (p->precision == B2P_FP64) return solve_T<double>(ctx, w, p, x0, y0, r, x_out, y_out);
    return solve_T<float>(ctx, w, p, x0, y0, r, x_out, y_out);
}

}  // namespace b2p
