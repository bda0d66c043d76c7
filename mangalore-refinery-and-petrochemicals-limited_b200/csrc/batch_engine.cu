// Batched engine: thousands of independent LPs in one persistent launch.
//
// Layout in HBM
//   * `nmat` constraint matrices concatenated into one block-diagonal CSR with
//     GLOBAL row/column indices (row_off[k], col_off[k] per matrix) plus its
//     stable transpose (FP64 originals and scaled copies: the restart-check KKT
//     and the re-centring read these).  Rows and columns of every matrix are
//     renumbered at upload by decreasing length (stable), so that consecutive
//     32-row / 32-column slices hold rows of nearly equal length.
//   * the iteration SpMVs read SELL-32 copies of the scaled matrix, one per
//     orientation: per slice of 32 rows (columns), `len` = the longest row of the
//     slice, entries stored column-major inside the slice (entry q of lane l at
//     slice_ptr + 32 q + l, zero-padded), values in the solve's precision and
//     16-bit LOCAL indices (an instance whose iterates fit in shared memory has
//     m, n < 65536).  A warp reads 32 consecutive values and 32 consecutive
//     indices per step: coalesced, no per-row pointers, no divergence.
//   * `count` instances, each naming a matrix; b, c, l, u in FP64 (internal
//     order; KKT and re-centring); per column one packed record {scaled cost,
//     lower, upper, Halpern anchor} and per row one {scaled rhs, dual lower
//     bound, anchor} in the solve's precision (16 bytes each in FP32: one
//     vector load); iterates x, y and the check-point copies xt, yt.  All
//     concatenated at x_off[i] / y_off[i]; warm starts and answers are mapped
//     between external and internal order on the device.
// Execution
//   * one CTA owns one instance at a time (persistent grid, work queue sorted by
//     nnz descending = longest-first) -- or, in the paired form for batches whose
//     instances share one matrix, two instances iterated in lockstep so that each
//     SELL load feeds both.  When a CTA takes an instance it copies its matrix's
//     slice pointers into a shared-memory table.  The gathered operands of both SpMVs --
//     y (also the dual iterate) for A^T y and xh for A xh -- live in shared
//     memory; x and the packed records stay in global memory, touched only by
//     their owning thread.  A PDHG iteration is: primal phase (one thread per
//     column, one warp per column slice) | barrier | dual phase (one thread per
//     row) | barrier.  A slice longer than kLongSlice entries per lane is summed
//     by the whole warp over the CSR copy instead (one dense row cannot stall
//     its slice).  Control scalars are private copies in every thread; the CTA
//     only meets in shared memory at restart-check iterations.
//   * precision MT (float = mixed, double = FP64) is the type of the scaled
//     matrix values, the packed records, the iterates and the SpMV sums.  FP64 is
//     kept for the scaling factors, the squared-residual sums, the KKT of the
//     original instance every K iterations, and the re-centring: the mixed
//     engine starts every restart epoch at an FP64 centre (xbar, ybar) and
//     solves the shifted problem rhs b - A xbar, cost c + A^T ybar, bounds
//     l - xbar, u - xbar, dual bound -ybar, rebuilt from the FP64 matrix, so
//     the FP32 iterates only carry the correction (iterative refinement).
//   * per instance: own step size (from its matrix), primal weight, Halpern
//     counter, restart state, FP64 KKT every K iterations (over FP64 SELL copies
//     with the checked vectors staged in shared memory; block reductions in a
//     fixed order: deterministic), own termination.
//   * a launch runs every active instance for up to `chunk` iterations; a
//     compaction kernel drops finished instances; [chunk, compact] x 2 is
//     captured as a CUDA graph and replayed until no instance is active.
//   * CTA size, SELL entry order (one entry or a pair per lane load), form
//     (single or paired) and chunk length come from an autotuner that times the
//     candidates on a sample of the batch (cached on disk).
#include <cub/cub.cuh>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>

#include "b2p_internal.cuh"

namespace b2p {

// per-instance control scalars (device)
struct InstCtrl {
    double omega, r0, rprev;
    double rel_p, rel_d, rel_g, pobj, dobj;
    double obj_err;  // FP64 bound on |c.x - optimum| / max(1, |c.x|) at the last check
    long long k, total, restarts;
    long long base;  // iterations spent on the instance before this run (cold fallback after a warm run)
    int status, done, first;
    int pad;
};

struct BatchWork {
    int nmat = 0, count = 0;
    int64_t tot_m = 0, tot_n = 0, nnz = 0, inst_m = 0, inst_n = 0;
    // matrices (internal numbering)
    DBuf<int32_t> rowptr, colidx, t_rowptr, t_colidx;
    DBuf<double> vals, t_vals, sv64, stv64, dr, dc, pv, pu;
    DBuf<float> sv32, stv32;
    DBuf<int32_t> mat_m, mat_n;
    DBuf<int64_t> mat_row_off, mat_col_off;
    DBuf<double> mat_eta;
    // SELL-32 copies: slice pointers (per matrix nslices + 1, at mat_*s_off), local
    // indices, scaled values in both precisions; internal -> external local index
    DBuf<int64_t> r_sptr, c_sptr, mat_rs_off, mat_cs_off;
    DBuf<uint16_t> r_eidx, c_eidx;
    DBuf<double> r_ev64, c_ev64;
    DBuf<float> r_ev32, c_ev32;
    DBuf<int32_t> r_ext, c_ext;
    std::vector<int32_t> h_mat_m, h_mat_n;
    // instances
    DBuf<int32_t> inst_mat;
    DBuf<int64_t> x_off, y_off;
    DBuf<double> b, c, lb, ub, bnorm, cnorm;
    DBuf<uint8_t> is_eq;
    // packed records and iterates, sized for FP64 and reinterpreted for FP32; dx, dy hold
    // the fixed-point displacement T(z) - z of the last check (infeasibility certificates)
    DBuf<double> colp, rowp, x, xt, y, yt, dx, dy;
    bool recenter = false;
    DBuf<double> xbar, atybar, ybar, axbar;  // re-centring state (per instance, original space)
    DBuf<InstCtrl> ictrl;
    DBuf<int32_t> active, active2, counters;  // counters[0]=head, [1]=active count
    std::vector<int32_t> h_inst_mat, order;
    int max_m = 0, max_n = 0;
    // results of the last solve: per-instance control blocks (host) and the answers
    // in the original space, external order (device, FP64), with the primal weights
    std::vector<InstCtrl> hc;
    DBuf<double> ox, oy, oom;
    bool solved = false;
    int tuned_threads[2] = {0, 0};  // block size per precision (0 = not tuned yet)
    int tuned_chunk[2] = {2048, 2048};  // iterations per chunk launch per precision
    int tuned_w[2] = {1, 1};        // SELL entry order per precision
    int tuned_ni[2] = {1, 1};       // instances per CTA per precision (2: paired form)
    int ell_w = 1;                  // entry order the SELL copies hold now
    DBuf<int32_t> list;             // instances re-initialised by a subset solve
    // active-instance trace of the last solve: host time (ms from the first graph launch of
    // the solve) and instances still active after each graph launch (a fallback run continues
    // the same trace)
    std::vector<double> trace_ms;
    std::vector<int32_t> trace_active;
};

void batch_free(Ctx* ctx) {
    delete ctx->bw;
    ctx->bw = nullptr;
}

namespace {

constexpr int kLongSlice = 128;  // entries per lane above which a slice is summed warp-cooperatively

// Packed per-column / per-row parameters of the scaled (and, when re-centred,
// shifted) problem in the solve's precision.
template <typename T>
struct alignas(4 * sizeof(T)) ColP {
    T c, l, u, a;  // cost, lower bound, upper bound, Halpern anchor
};
template <typename T>
struct alignas(4 * sizeof(T)) RowP {
    T b, lo, a, pad;  // rhs, lower bound of the dual (-inf on equality rows), anchor
};

struct BArgs {
    // matrices
    const int32_t *rowptr, *colidx, *t_rowptr, *t_colidx;
    const double *sv64, *stv64, *dr, *dc, *mat_eta;
    const void *sv, *stv;  // MT-typed scaled values (CSR)
    const int32_t *mat_m, *mat_n;
    const int64_t *mat_row_off, *mat_col_off;
    // SELL-32 copies
    const int64_t *r_sptr, *c_sptr, *mat_rs_off, *mat_cs_off;
    const uint16_t *r_eidx, *c_eidx;
    const void *r_ev, *c_ev;  // MT-typed
    const double *r_ev64, *c_ev64;  // FP64 values in the same order (restart-check KKT)
    const int32_t *r_ext, *c_ext;
    // instances
    const int32_t* inst_mat;
    const int64_t *x_off, *y_off;
    const double *b, *c, *lb, *ub;
    double *bnorm, *cnorm;  // written by the init kernel
    const uint8_t* is_eq;
    void *colp, *rowp, *x, *xt, *y, *yt;  // MT-typed
    void *dx, *dy;                        // MT-typed: T(z) - z at check iterations (eps_inf > 0)
    InstCtrl* ictrl;
    const int32_t* active;
    int32_t* counters;
    // parameters
    double eps, beta_s, beta_n, beta_a, rho;
    double eps_obj, eps_inf;  // objective-accuracy stop (0 = off), certificate tolerance (0 = off)
    // FP64 re-centring: per-instance centre in the original space, A xbar, A^T ybar;
    // original FP64 values in both orientations
    int recenter;
    const double *vals, *t_vals;
    double *xbar, *ybar, *axbar, *atybar;
    long long max_iter;
    int K;
};

template <typename T>
__device__ __forceinline__ T clampT(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Block-wide FP64 sum of NV values (sh holds 32 * NV), fixed reduction order (deterministic).
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* sh /* [32*NV] */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[w * NV + q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double t = 0.0;
            for (int i = 0; i < nw; ++i) t += sh[i * NV + q];
            v[q] = t;
        }
    }
}

// One lane's row of a SELL-32 slice (len entries per lane, even).  W = 1: v / ix point at
// the lane's first entry and entry q sits 32 q further.  W = 2: entries are stored in
// pairs -- pair t of lane l at slice + 64 t + 2 l -- so one 8- (FP32) or 16-byte (FP64)
// value load and one 4-byte index load fetch two entries; v / ix point at the lane's
// first pair.  Sequential sum in entry order in both layouts (bit-identical results).
// Entries are taken in batches of B (8 in FP32, 4 in FP64, the most the register
// budget of two 512-thread CTAs per SM holds without spilling in the loop): every
// value and index load of a batch (the last batch predicated on the row's length)
// is issued before the first gather that needs one, so a slice of up to B entries
// per lane costs one L2 round trip and a longer one a round trip per batch.
template <typename VT, typename GT, int W>
__device__ __forceinline__ VT ell_dot_vg(const VT* __restrict__ v, const uint16_t* __restrict__ ix, int len,
                                        const GT* __restrict__ g) {
    constexpr int B = sizeof(VT) == 4 ? 8 : 4;
    VT s = (VT)0;
    if constexpr (W == 1) {
        for (int q = 0; q < len; q += B) {
            VT vv[B];
            unsigned ii[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const bool h = q + u < len;
                vv[u] = h ? v[(q + u) * 32] : (VT)0;
                ii[u] = h ? (unsigned)ix[(q + u) * 32] : 0u;
            }
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (q + u < len) s += vv[u] * (VT)g[ii[u]];
        }
    } else {
        typedef typename std::conditional<sizeof(VT) == 4, float2, double2>::type VT2;
        constexpr int P = B / 2;  // pairs per batch
        const int np = len >> 1;
        for (int t = 0; t < np; t += P) {
            VT2 vv[P];
            unsigned ii[P];
#pragma unroll
            for (int u = 0; u < P; ++u) {
                const bool h = t + u < np;
                vv[u] = h ? *reinterpret_cast<const VT2*>(v + (t + u) * 64) : VT2{(VT)0, (VT)0};
                ii[u] = h ? *reinterpret_cast<const unsigned*>(ix + (t + u) * 64) : 0u;
            }
#pragma unroll
            for (int u = 0; u < P; ++u)
                if (t + u < np) {
                    s += vv[u].x * (VT)g[ii[u] & 0xFFFFu];
                    s += vv[u].y * (VT)g[ii[u] >> 16];
                }
        }
    }
    return s;
}

template <typename MT, int W>
__device__ __forceinline__ MT ell_dot(const MT* __restrict__ v, const uint16_t* __restrict__ ix, int len,
                                      const MT* __restrict__ g) {
    return ell_dot_vg<MT, MT, W>(v, ix, len, g);
}

// ell_dot for two instances of one matrix: every value and index load of the slice
// feeds a gather from each instance's operand (g0, g1) and two independent sums, each
// in the entry order of ell_dot (the same results as two ell_dot calls).
template <typename MT, int W>
__device__ __forceinline__ void ell_dot2(const MT* __restrict__ v, const uint16_t* __restrict__ ix, int len,
                                         const MT* __restrict__ g0, const MT* __restrict__ g1, MT& s0, MT& s1) {
    constexpr int B = sizeof(MT) == 4 ? 8 : 4;
    MT a0 = (MT)0, a1 = (MT)0;
    if constexpr (W == 1) {
        for (int q = 0; q < len; q += B) {
            MT vv[B];
            unsigned ii[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const bool h = q + u < len;
                vv[u] = h ? v[(q + u) * 32] : (MT)0;
                ii[u] = h ? (unsigned)ix[(q + u) * 32] : 0u;
            }
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (q + u < len) {
                    a0 += vv[u] * g0[ii[u]];
                    a1 += vv[u] * g1[ii[u]];
                }
        }
    } else {
        typedef typename std::conditional<sizeof(MT) == 4, float2, double2>::type MT2;
        constexpr int P = B / 2;
        const int np = len >> 1;
        for (int t = 0; t < np; t += P) {
            MT2 vv[P];
            unsigned ii[P];
#pragma unroll
            for (int u = 0; u < P; ++u) {
                const bool h = t + u < np;
                vv[u] = h ? *reinterpret_cast<const MT2*>(v + (t + u) * 64) : MT2{(MT)0, (MT)0};
                ii[u] = h ? *reinterpret_cast<const unsigned*>(ix + (t + u) * 64) : 0u;
            }
#pragma unroll
            for (int u = 0; u < P; ++u)
                if (t + u < np) {
                    const unsigned lo = ii[u] & 0xFFFFu, hi = ii[u] >> 16;
                    a0 += vv[u].x * g0[lo];
                    a1 += vv[u].x * g1[lo];
                    a0 += vv[u].y * g0[hi];
                    a1 += vv[u].y * g1[hi];
                }
        }
    }
    s0 = a0;
    s1 = a1;
}

// Entries of a CTA's slice table (column slices, then row slices; even, so what follows
// it in shared memory stays 16-byte aligned).
__host__ __device__ __forceinline__ int slice_tab_len(int nrs, int ncs) { return (nrs + ncs + 1) & ~1; }

// The slice table of one matrix in shared memory, built when a CTA takes an instance:
// per slice {first entry, entries per lane}.  The iterations then read one 8-byte shared
// word per slice instead of two slice pointers from L2 in front of every value load.
// Entry offsets fit 32 bits (the upload refuses batches whose SELL copies do not).
__device__ __forceinline__ void fill_slice_tab(int2* tab, const int64_t* __restrict__ csp, int ncs,
                                               const int64_t* __restrict__ rsp, int nrs) {
    for (int i = threadIdx.x; i < ncs; i += blockDim.x)
        tab[i] = make_int2((int)csp[i], (int)((csp[i + 1] - csp[i]) >> 5));
    for (int i = threadIdx.x; i < nrs; i += blockDim.x)
        tab[ncs + i] = make_int2((int)rsp[i], (int)((rsp[i + 1] - rsp[i]) >> 5));
}

// Slice of round r for warp w of nw: rounds alternate the direction in which the
// (length-sorted) slices are dealt, w then nw - 1 - w, so every warp's share of long
// and short slices is even.  Increasing in r for a fixed warp.
__device__ __forceinline__ int snake_slice(int r, int w, int nw) { return r * nw + ((r & 1) ? nw - 1 - w : w); }

// The 32 rows of one slice summed by the whole warp over the CSR copy (rows
// first .. first+cnt-1, global numbering; `off` localises the column index).
// Lane r returns the sum of row first + r.
template <typename MT, typename GT = MT>
__device__ MT long_slice_dot(const MT* __restrict__ vals, const int32_t* __restrict__ ptr,
                             const int32_t* __restrict__ idx, int64_t first, int cnt, int64_t off,
                             const GT* __restrict__ g, int lane) {
    MT mine = (MT)0;
    for (int r = 0; r < cnt; ++r) {
        MT s = (MT)0;
        for (int e = ptr[first + r] + lane; e < ptr[first + r + 1]; e += 32) s += vals[e] * (MT)g[idx[e] - off];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == r) mine = s;
    }
    return mine;
}

// Re-centring, an exact change of variables in FP64: rewrite the scaled problem of
// one instance around its centre (xbar, ybar) -- rhs dr*(b - A xbar), cost
// dc*(c + A^T ybar), bounds (l - xbar)/dc, (u - xbar)/dc, dual lower bound -ybar/dr
// on inequality rows -- from the original FP64 matrix, with zero anchors (the
// iterates restart at the centre).  Called by every thread of the owning CTA.
template <typename MT>
__device__ void rebuild_shifted(const BArgs& a, int m, int n, int64_t ro, int64_t co, int64_t xo, int64_t yo) {
    ColP<MT>* colp = (ColP<MT>*)a.colp;
    RowP<MT>* rowp = (RowP<MT>*)a.rowp;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int64_t gi = ro + i;
        double s = 0.0;
        for (int e = a.rowptr[gi]; e < a.rowptr[gi + 1]; ++e) s += a.vals[e] * a.xbar[xo + a.colidx[e] - co];
        const double dri = a.dr[gi];
        a.axbar[yo + i] = s;
        RowP<MT> r;
        r.b = (MT)(dri * (a.b[yo + i] - s));
        r.lo = a.is_eq[yo + i] ? (MT)(-INFINITY) : (MT)(-a.ybar[yo + i] / dri);
        r.a = (MT)0;
        r.pad = (MT)0;
        rowp[yo + i] = r;
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const int64_t gj = co + j;
        double s = 0.0;
        for (int e = a.t_rowptr[gj]; e < a.t_rowptr[gj + 1]; ++e) s += a.t_vals[e] * a.ybar[yo + a.t_colidx[e] - ro];
        const double dcj = a.dc[gj], xb = a.xbar[xo + j];
        a.atybar[xo + j] = s;
        ColP<MT> p;
        p.c = (MT)(dcj * (a.c[xo + j] + s));
        p.l = (MT)((a.lb[xo + j] - xb) / dcj);
        p.u = (MT)((a.ub[xo + j] - xb) / dcj);
        p.a = (MT)0;
        colp[xo + j] = p;
    }
}

// Restart of one instance after its check decided so, by every thread of the owning
// CTA (ys: its dual iterate in shared memory): z <- anchor <- T(z), or, re-centred,
// T(z) becomes the new FP64 centre and the shifted problem is rebuilt around it.
template <typename MT>
__device__ __forceinline__ void restart_instance(const BArgs& a, int m, int n, int64_t ro, int64_t co, int64_t xo,
                                              int64_t yo, MT* ys) {
    const int tid = threadIdx.x, nt = blockDim.x;
    ColP<MT>* colp = (ColP<MT>*)a.colp;
    RowP<MT>* rowp = (RowP<MT>*)a.rowp;
    MT *xg = (MT*)a.x, *xtg = (MT*)a.xt, *ytg = (MT*)a.yt;
    if (!a.recenter) {
        for (int j = tid; j < n; j += nt) {
            const MT v = xtg[xo + j];
            xg[xo + j] = v;
            colp[xo + j].a = v;
        }
        for (int i = tid; i < m; i += nt) {
            const MT v = ytg[yo + i];
            ys[i] = v;
            rowp[yo + i].a = v;
        }
    } else {
        for (int j = tid; j < n; j += nt) {
            a.xbar[xo + j] += a.dc[co + j] * (double)xtg[xo + j];
            xg[xo + j] = (MT)0;
            xtg[xo + j] = (MT)0;
        }
        for (int i = tid; i < m; i += nt) {
            a.ybar[yo + i] += a.dr[ro + i] * (double)ytg[yo + i];
            ys[i] = (MT)0;
            ytg[yo + i] = (MT)0;
        }
        __syncthreads();
        rebuild_shifted<MT>(a, m, n, ro, co, xo, yo);
    }
}

// Restart-check iteration of one instance, run by every thread of the owning CTA
// after T(z) (xt, yt) and, with certificates on, the displacement (dx, dy) are in
// global memory: the FP64 KKT of T(z) on the original instance, the objective-error
// bound, the certificates (every fourth check) and the decisions -- termination,
// restart, primal weight -- which thread 0 writes to `sc` and `s_flags` (0: done,
// 1: restart).  The products A xt, A^T yt (and A dx, A^T dy) run over the FP64 SELL
// copies of the scaled matrix with the slice table `tab`, one lane per row / column as
// in the iterations, gathering from `buf` -- the instance's xh region of shared memory,
// free at a check (the dual phase has consumed xh, the next primal phase rewrites it) --
// into which each gathered vector is staged first.  Kept out of line: its FP64
// accumulators would otherwise raise the register demand of the iteration loop.
template <typename MT, int W>
__device__ __noinline__ void check_instance(const BArgs& a, int inst, int m, int n, int64_t ro, int64_t co,
                                            int64_t xo, int64_t yo, long long total, long long kk, double om,
                                            double r_now, double dxa, double dya, InstCtrl& sc, int* s_flags,
                                            double* red, const int2* tab, MT* buf) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const int ncs = (n + 31) >> 5, nrs = (m + 31) >> 5;
    const MT *xtg = (const MT*)a.xt, *ytg = (const MT*)a.yt;
    const MT *dxg = (const MT*)a.dx, *dyg = (const MT*)a.dy;
    const bool rays = a.eps_inf > 0.0;
    // (A v)_i in the scaled space for lane `lane` of row slice sl, v staged in buf
    auto row_dot = [&](int sl) -> double {
        const int2 t = tab[ncs + sl];
        return t.y <= kLongSlice
                   ? ell_dot_vg<double, MT, W>(a.r_ev64 + t.x + W * lane, a.r_eidx + t.x + W * lane, t.y, buf)
                   : long_slice_dot<double, MT>(a.sv64, a.rowptr, a.colidx, ro + (sl << 5), min(32, m - (sl << 5)),
                                                co, buf, lane);
    };
    auto col_dot = [&](int sl) -> double {
        const int2 t = tab[sl];
        return t.y <= kLongSlice
                   ? ell_dot_vg<double, MT, W>(a.c_ev64 + t.x + W * lane, a.c_eidx + t.x + W * lane, t.y, buf)
                   : long_slice_dot<double, MT>(a.stv64, a.t_rowptr, a.t_colidx, co + (sl << 5),
                                                min(32, n - (sl << 5)), ro, buf, lane);
    };
    // ---- FP64 KKT of T(z) on the original instance and the objective-error bound
    double kk2[6] = {0, 0, 0, 0, 0, 0};
    // |primal residual|^2, b.y, |dual residual|^2, c.x, bound term, sum |y| viol
    for (int j = tid; j < n; j += nt) buf[j] = xtg[xo + j];
    __syncthreads();
    for (int sl = warp; sl < nrs; sl += nwarps) {
        const int i = (sl << 5) + lane;
        const double s = row_dot(sl);
        if (i < m) {
            const double dri = a.dr[ro + i];
            const double ax = (a.recenter ? a.axbar[yo + i] : 0.0) + s / dri;
            double rp = ax - a.b[yo + i];
            if (!a.is_eq[yo + i]) rp = fmax(rp, 0.0);
            kk2[0] += rp * rp;
            const double yv = (a.recenter ? a.ybar[yo + i] : 0.0) + dri * (double)ytg[yo + i];
            kk2[1] += a.b[yo + i] * yv;
            kk2[5] += fabs(yv) * fabs(rp);
            if (!a.is_eq[yo + i] && yv < 0.0) kk2[2] += yv * yv;  // y >= 0 on <= rows (dual residual)
        }
    }
    __syncthreads();  // every warp is done with xt
    for (int i = tid; i < m; i += nt) buf[i] = ytg[yo + i];
    __syncthreads();
    for (int sl = warp; sl < ncs; sl += nwarps) {
        const int j = (sl << 5) + lane;
        const double s = col_dot(sl);
        if (j < n) {
            const double dcj = a.dc[co + j];
            const double cj = a.c[xo + j], lj = a.lb[xo + j], uj = a.ub[xo + j];
            const double g = cj + (a.recenter ? a.atybar[xo + j] : 0.0) + s / dcj;
            const bool fl = isfinite(lj), fu = isfinite(uj);
            const double lam = (fl && fu) ? g : (fl ? fmax(g, 0.0) : (fu ? fmin(g, 0.0) : 0.0));
            const double rd = g - lam;
            kk2[2] += rd * rd;
            kk2[3] += cj * ((a.recenter ? a.xbar[xo + j] : 0.0) + dcj * (double)xtg[xo + j]);
            if (lam > 0.0) kk2[4] += lam * lj;
            else if (lam < 0.0) kk2[4] += lam * uj;
        }
    }
    block_sums<6>(kk2, red);
    // ---- certificates of the displacement dx, dy = T(z) - z (every fourth check): primal
    // ray dx -- 0 |viol of A dx and of the bounds' recession cone|^2, 1 c.dx, 2 sum |c dx|;
    // dual ray dy -- 3 b.dy, 4 bound term of a = A^T dy, 5 sum of |terms|, 6 |viol of a|^2
    double ry[7] = {0, 0, 0, 0, 0, 0, 0};
    const bool ray_check = rays && ((total / a.K) & 3) == 0;
    if (ray_check) {
        for (int j = tid; j < n; j += nt) buf[j] = dxg[xo + j];
        __syncthreads();
        for (int sl = warp; sl < nrs; sl += nwarps) {
            const int i = (sl << 5) + lane;
            const double s = row_dot(sl);
            if (i < m) {
                const double dri = a.dr[ro + i];
                const double adx = s / dri;  // (A dx)_i in the original space
                const double v = a.is_eq[yo + i] ? adx : fmax(adx, 0.0);
                ry[0] += v * v;
                const double dyo = dri * (double)dyg[yo + i];
                ry[3] += a.b[yo + i] * dyo;
                ry[5] += fabs(a.b[yo + i] * dyo);
            }
        }
        __syncthreads();
        for (int i = tid; i < m; i += nt) buf[i] = dyg[yo + i];
        __syncthreads();
        for (int sl = warp; sl < ncs; sl += nwarps) {
            const int j = (sl << 5) + lane;
            const double s = col_dot(sl);
            if (j < n) {
                const double dcj = a.dc[co + j];
                const double cj = a.c[xo + j], lj = a.lb[xo + j], uj = a.ub[xo + j];
                const bool fl = isfinite(lj), fu = isfinite(uj);
                const double dxo = dcj * (double)dxg[xo + j];
                ry[1] += cj * dxo;
                ry[2] += fabs(cj * dxo);
                const double bv = (fl && dxo < 0.0 ? -dxo : 0.0) + (fu && dxo > 0.0 ? dxo : 0.0);
                ry[0] += bv * bv;
                const double at = s / dcj;  // (A^T dy)_j in the original space
                const double t = at > 0.0 ? (fl ? at * lj : 0.0) : (at < 0.0 ? (fu ? at * uj : 0.0) : 0.0);
                ry[4] += t;
                ry[5] += fabs(t);
                const double av = (!fl && at > 0.0 ? at : 0.0) + (!fu && at < 0.0 ? -at : 0.0);
                ry[6] += av * av;
            }
        }
        block_sums<7>(ry, red);
    }
    if (tid == 0) {
        const double pres = sqrt(kk2[0]), dres = sqrt(kk2[2]);
        const double pobj = kk2[3], dobj = -kk2[1] + kk2[4];
        sc.rel_p = pres / (1.0 + a.bnorm[inst]);
        sc.rel_d = dres / (1.0 + a.cnorm[inst]);
        sc.rel_g = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
        sc.pobj = pobj;
        sc.dobj = dobj;
        sc.obj_err = fmax(fmax(pobj - dobj, kk2[5]), 0.0) / fmax(1.0, fabs(pobj));
        const bool finite = isfinite(pres) && isfinite(dres) && isfinite(pobj) && isfinite(dobj) && isfinite(r_now);
        const bool obj_ok = a.eps_obj <= 0.0 || sc.obj_err <= a.eps_obj;
        // certificates (ratio tests of PDLP; the 1e-9 floors keep rounding noise of a
        // vanishing displacement from passing for a ray)
        const double dray = -ry[3] + ry[4], pray = ry[1];
        const bool infeas = ray_check && dray > 0.0 && dray > 1e-9 * ry[5] && sqrt(ry[6]) <= a.eps_inf * dray;
        const bool unbnd = ray_check && pray < 0.0 && -pray > 1e-9 * ry[2] && sqrt(ry[0]) <= a.eps_inf * -pray;
        if (!finite) {
            sc.done = 1;
            sc.status = B2P_STATUS_NUMERICAL_FAILURE;
        } else if (sc.rel_p <= a.eps && sc.rel_d <= a.eps && sc.rel_g <= a.eps && obj_ok) {
            sc.done = 1;
            sc.status = B2P_STATUS_OPTIMAL;
        } else if (infeas) {
            sc.done = 1;
            sc.status = B2P_STATUS_INFEASIBLE_DETECTED;
        } else if (unbnd) {
            sc.done = 1;
            sc.status = B2P_STATUS_UNBOUNDED_DETECTED;
        } else if (total + sc.base >= a.max_iter) {
            sc.done = 1;
            sc.status = B2P_STATUS_MAX_ITERATIONS;
        }
        s_flags[1] = 0;
        if (!sc.done) {
            const bool rs = (r_now <= a.beta_s * sc.r0) || (r_now <= a.beta_n * sc.r0 && r_now > sc.rprev) ||
                            ((double)kk >= a.beta_a * (double)total);
            sc.rprev = r_now;
            if (rs) {
                if (dxa > 1e-10 && dya > 1e-10) {
                    const double nw = exp(0.5 * log(dya / dxa) + 0.5 * log(om));
                    if (isfinite(nw) && nw > 0.0) sc.omega = nw;
                }
                sc.restarts += 1;
                s_flags[1] = 1;
            }
        }
        s_flags[0] = sc.done;
    }
}

// Body of the persistent chunk kernel; launched as k_batch_chunk (the tuned CTA
// size, up to 512 threads, two CTAs per SM) while many instances are active and as
// k_batch_chunk_wide (1024 threads, one CTA per SM) once no more than one instance
// per SM is left, so the last, slowest instances iterate with twice the threads.
template <typename MT, int W>
__device__ __forceinline__ void batch_chunk_body(const BArgs& a, int chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32 * 7];
    __shared__ InstCtrl sc;
    __shared__ int s_q;
    __shared__ int s_flags[2];  // 0: done, 1: restart
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const MT* sv = (const MT*)a.sv;
    const MT* stv = (const MT*)a.stv;
    const MT* rev = (const MT*)a.r_ev;
    const MT* cev = (const MT*)a.c_ev;
    ColP<MT>* colp = (ColP<MT>*)a.colp;
    RowP<MT>* rowp = (RowP<MT>*)a.rowp;
    MT *xg = (MT*)a.x, *xtg = (MT*)a.xt, *yg = (MT*)a.y, *ytg = (MT*)a.yt;
    MT *dxg = (MT*)a.dx, *dyg = (MT*)a.dy;
    const bool rays = a.eps_inf > 0.0;
    const int active_count = a.counters[1];
    const MT rho = (MT)a.rho, one_rho = (MT)(1.0 + a.rho);
    while (true) {
        if (tid == 0) s_q = atomicAdd(&a.counters[0], 1);
        __syncthreads();
        const int q = s_q;
        if (q >= active_count) break;
        const int inst = a.active[q];
        const int mat = a.inst_mat[inst];
        const int m = a.mat_m[mat], n = a.mat_n[mat];
        const int64_t ro = a.mat_row_off[mat], co = a.mat_col_off[mat];
        const int64_t xo = a.x_off[inst], yo = a.y_off[inst];
        const int64_t* rsp = a.r_sptr + a.mat_rs_off[mat];
        const int64_t* csp = a.c_sptr + a.mat_cs_off[mat];
        const int nrs = (m + 31) >> 5, ncs = (n + 31) >> 5;
        const double eta = a.mat_eta[mat];
        int2* tab = (int2*)smem_raw;  // column slices, then row slices
        MT* ys = (MT*)(tab + slice_tab_len(nrs, ncs));
        MT* xhs = ys + ((m + 3) & ~3);
        fill_slice_tab(tab, csp, ncs, rsp, nrs);
        if (tid == 0) sc = a.ictrl[inst];
        for (int i = tid; i < m; i += nt) ys[i] = yg[yo + i];
        __syncthreads();
        long long kk = sc.k, total = sc.total;
        bool first = sc.first != 0;
        double om = sc.omega;
        __syncthreads();  // every thread holds its copy before thread 0 writes sc again
        bool done = false;
        for (int it = 0; it < chunk && !done; ++it) {
            const bool check = ((total + 1) % a.K) == 0;
            const bool stats = first || check;
            const MT tau = (MT)(eta / om), sigma = (MT)(eta * om);
            const MT wk = (MT)((kk + 1.0) / (kk + 2.0)), wa = (MT)(1.0 / (kk + 2.0));
            double acc[4] = {0, 0, 0, 0};  // |x - T(x)|^2 and |y - T(y)|^2 (first or check), distances to anchors
            // ---- primal phase: one thread per column, gathers y from shared memory; slices
            // (longest first) are dealt to the warps boustrophedon-wise, which evens out the
            // warps' load round trips before the barrier
            for (int r = 0, sl = warp; sl < ncs; ++r, sl = snake_slice(r, warp, nwarps)) {
                const int j = (sl << 5) + lane;
                const bool valid = j < n;
                ColP<MT> p;
                MT x0 = (MT)0;
                if (valid) {
                    p = colp[xo + j];
                    x0 = xg[xo + j];
                }
                const int2 t = tab[sl];
                const int p0 = t.x, len = t.y;
                const MT s = len <= kLongSlice
                                 ? ell_dot<MT, W>(cev + p0 + W * lane, a.c_eidx + p0 + W * lane, len, ys)
                                 : long_slice_dot<MT>(stv, a.t_rowptr, a.t_colidx, co + (sl << 5), min(32, n - (sl << 5)),
                                                      ro, ys, lane);
                if (valid) {
                    const MT xt = clampT(x0 - tau * (p.c + s), p.l, p.u);
                    xhs[j] = (MT)2 * xt - x0;
                    xg[xo + j] = wk * (one_rho * xt - rho * x0) + wa * p.a;
                    if (stats) {
                        const double d = (double)x0 - (double)xt;
                        acc[0] += d * d;
                    }
                    if (check) {
                        xtg[xo + j] = xt;
                        if (rays) dxg[xo + j] = xt - x0;
                        const double e = (double)xt - (double)p.a;
                        acc[1] += e * e;
                    }
                }
            }
            __syncthreads();
            // ---- dual phase: one thread per row, gathers xh from shared memory
            for (int r = 0, sl = warp; sl < nrs; ++r, sl = snake_slice(r, warp, nwarps)) {
                const int i = (sl << 5) + lane;
                const bool valid = i < m;
                RowP<MT> p;
                if (valid) p = rowp[yo + i];
                const int2 t = tab[ncs + sl];
                const int p0 = t.x, len = t.y;
                const MT s = len <= kLongSlice
                                 ? ell_dot<MT, W>(rev + p0 + W * lane, a.r_eidx + p0 + W * lane, len, xhs)
                                 : long_slice_dot<MT>(sv, a.rowptr, a.colidx, ro + (sl << 5), min(32, m - (sl << 5)),
                                                      co, xhs, lane);
                if (valid) {
                    const MT y0 = ys[i];
                    MT yt = y0 + sigma * (s - p.b);
                    if (yt < p.lo) yt = p.lo;  // NaN stays NaN
                    ys[i] = wk * (one_rho * yt - rho * y0) + wa * p.a;
                    if (stats) {
                        const double d = (double)y0 - (double)yt;
                        acc[2] += d * d;
                    }
                    if (check) {
                        ytg[yo + i] = yt;
                        if (rays) {  // a dual ray candidate keeps y >= 0 on <= rows (p.lo = -inf on = rows)
                            MT d = yt - y0;
                            if (p.lo != (MT)(-INFINITY) && d < (MT)0) d = (MT)0;
                            dyg[yo + i] = d;
                        }
                        const double e = (double)yt - (double)p.a;
                        acc[3] += e * e;
                    }
                }
            }
            kk += 1;
            total += 1;
            if (!stats) {
                __syncthreads();
                continue;
            }
            block_sums<4>(acc, red);
            const bool was_first = first;
            first = false;
            if (!check) {  // first iteration after a (re)start: the restart reference residual
                if (tid == 0) {
                    sc.r0 = sqrt(om * acc[0] + acc[2] / om);
                    sc.rprev = sc.r0;
                }
                __syncthreads();
                continue;
            }
            double r_now = 0, dxa = 0, dya = 0;
            if (tid == 0) {
                r_now = sqrt(om * acc[0] + acc[2] / om);
                if (was_first) {
                    sc.r0 = r_now;
                    sc.rprev = r_now;
                }
                dxa = sqrt(acc[1]);
                dya = sqrt(acc[3]);
            }
            __syncthreads();  // xt / yt of this iteration are in global memory
            check_instance<MT, W>(a, inst, m, n, ro, co, xo, yo, total, kk, om, r_now, dxa, dya, sc, s_flags, red,
                                  tab, xhs);
            __syncthreads();
            done = s_flags[0] != 0;
            om = sc.omega;
            if (s_flags[1]) {
                kk = 0;
                first = true;
                restart_instance<MT>(a, m, n, ro, co, xo, yo, ys);
            }
            __syncthreads();
        }
        // store the dual iterate and the control block
        for (int i = tid; i < m; i += nt) yg[yo + i] = ys[i];
        if (tid == 0) {
            sc.k = kk;
            sc.total = total;
            sc.first = first ? 1 : 0;
            a.ictrl[inst] = sc;
        }
        __syncthreads();
    }
}

template <typename MT, int W>
__global__ void __launch_bounds__(512, 2) k_batch_chunk(const __grid_constant__ BArgs a, int chunk) {
    batch_chunk_body<MT, W>(a, chunk);
}

template <typename MT, int W>
__global__ void __launch_bounds__(1024, 1) k_batch_chunk_wide(const __grid_constant__ BArgs a, int chunk) {
    batch_chunk_body<MT, W>(a, chunk);
}

// Paired form of the chunk kernel for a batch whose instances all share one matrix
// (a parametric family): a CTA takes two consecutive entries of the active list and
// iterates both instances in lockstep, so every SELL value and index load of the
// shared matrix feeds both instances' gathers (ell_dot2) -- the matrix bytes per
// instance-iteration halve and each warp carries two independent sums per load.
// Shared memory holds y and xh of both instances.  Per instance everything is as in
// batch_chunk_body, with the same thread-to-column/row assignment and arithmetic, so
// the iterates and decisions are those of the single form bit for bit.  An instance
// that finishes leaves its partner to iterate alone (single gathers) until the chunk
// ends; the compaction between chunks re-pairs the survivors.
template <typename MT, int W>
__device__ __forceinline__ void batch_pair_body(const BArgs& a, int chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32 * 7];
    __shared__ InstCtrl sc[2];
    __shared__ int s_q;
    __shared__ int s_flags[2][2];  // per instance -- 0: done, 1: restart
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const MT* sv = (const MT*)a.sv;
    const MT* stv = (const MT*)a.stv;
    const MT* rev = (const MT*)a.r_ev;
    const MT* cev = (const MT*)a.c_ev;
    ColP<MT>* colp = (ColP<MT>*)a.colp;
    RowP<MT>* rowp = (RowP<MT>*)a.rowp;
    MT *xg = (MT*)a.x, *xtg = (MT*)a.xt, *yg = (MT*)a.y, *ytg = (MT*)a.yt;
    MT *dxg = (MT*)a.dx, *dyg = (MT*)a.dy;
    const bool rays = a.eps_inf > 0.0;
    const int active_count = a.counters[1];
    const MT rho = (MT)a.rho, one_rho = (MT)(1.0 + a.rho);
    // the one matrix of the batch
    const int m = a.mat_m[0], n = a.mat_n[0];
    const int64_t ro = a.mat_row_off[0], co = a.mat_col_off[0];
    const int64_t* rsp = a.r_sptr + a.mat_rs_off[0];
    const int64_t* csp = a.c_sptr + a.mat_cs_off[0];
    const int nrs = (m + 31) >> 5, ncs = (n + 31) >> 5;
    const double eta = a.mat_eta[0];
    const int m4 = (m + 3) & ~3, stride = m4 + max((n + 3) & ~3, m4);  // xh region also stages y at checks
    int2* tab = (int2*)smem_raw;  // column slices, then row slices (built once: one matrix)
    MT* ysb[2] = {(MT*)(tab + slice_tab_len(nrs, ncs)), (MT*)(tab + slice_tab_len(nrs, ncs)) + stride};
    MT* xhb[2] = {ysb[0] + m4, ysb[1] + m4};
    fill_slice_tab(tab, csp, ncs, rsp, nrs);
    while (true) {
        if (tid == 0) s_q = atomicAdd(&a.counters[0], 2);
        __syncthreads();
        const int q = s_q;
        if (q >= active_count) break;
        const bool has2 = q + 1 < active_count;
        int inst[2];
        inst[0] = a.active[q];
        inst[1] = has2 ? a.active[q + 1] : inst[0];
        bool live[2] = {true, has2};
        int64_t xo[2], yo[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            xo[k] = a.x_off[inst[k]];
            yo[k] = a.y_off[inst[k]];
        }
        if (tid == 0) sc[0] = a.ictrl[inst[0]];
        if (tid == 1 && has2) sc[1] = a.ictrl[inst[1]];
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (live[k])
                for (int i = tid; i < m; i += nt) ysb[k][i] = yg[yo[k] + i];
        __syncthreads();
        long long kk[2], total[2];
        bool first[2];
        double om[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int src = live[k] ? k : 0;
            kk[k] = sc[src].k;
            total[k] = sc[src].total;
            first[k] = sc[src].first != 0;
            om[k] = sc[src].omega;
        }
        __syncthreads();  // every thread holds its copies before thread 0 writes sc again
        for (int it = 0; it < chunk && (live[0] || live[1]); ++it) {
            bool check[2], stats[2];
            MT tau[2], sigma[2], wk[2], wa[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                check[k] = live[k] && ((total[k] + 1) % a.K) == 0;
                stats[k] = live[k] && (first[k] || check[k]);
                tau[k] = (MT)(eta / om[k]);
                sigma[k] = (MT)(eta * om[k]);
                wk[k] = (MT)((kk[k] + 1.0) / (kk[k] + 2.0));
                wa[k] = (MT)(1.0 / (kk[k] + 2.0));
            }
            const bool both = live[0] && live[1];
            const bool solo1 = !live[0];  // the one live instance when not both
            const MT* ys_solo = solo1 ? ysb[1] : ysb[0];
            const MT* xh_solo = solo1 ? xhb[1] : xhb[0];
            double acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            // ---- primal phase
            for (int r = 0, sl = warp; sl < ncs; ++r, sl = snake_slice(r, warp, nwarps)) {
                const int j = (sl << 5) + lane;
                const bool valid = j < n;
                ColP<MT> p[2];
                MT x0[2] = {(MT)0, (MT)0};
#pragma unroll
                for (int k = 0; k < 2; ++k)
                    if (valid && live[k]) {
                        p[k] = colp[xo[k] + j];
                        x0[k] = xg[xo[k] + j];
                    }
                const int2 tb = tab[sl];
                const int p0 = tb.x, len = tb.y;
                MT s[2] = {(MT)0, (MT)0};
                if (len <= kLongSlice) {
                    if (both)
                        ell_dot2<MT, W>(cev + p0 + W * lane, a.c_eidx + p0 + W * lane, len, ysb[0], ysb[1], s[0], s[1]);
                    else {
                        const MT t = ell_dot<MT, W>(cev + p0 + W * lane, a.c_eidx + p0 + W * lane, len, ys_solo);
                        s[0] = solo1 ? (MT)0 : t;
                        s[1] = solo1 ? t : (MT)0;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        if (live[k])
                            s[k] = long_slice_dot<MT>(stv, a.t_rowptr, a.t_colidx, co + (sl << 5),
                                                      min(32, n - (sl << 5)), ro, ysb[k], lane);
                }
#pragma unroll
                for (int k = 0; k < 2; ++k)
                    if (valid && live[k]) {
                        const MT xt = clampT(x0[k] - tau[k] * (p[k].c + s[k]), p[k].l, p[k].u);
                        xhb[k][j] = (MT)2 * xt - x0[k];
                        xg[xo[k] + j] = wk[k] * (one_rho * xt - rho * x0[k]) + wa[k] * p[k].a;
                        if (stats[k]) {
                            const double d = (double)x0[k] - (double)xt;
                            acc[k][0] += d * d;
                        }
                        if (check[k]) {
                            xtg[xo[k] + j] = xt;
                            if (rays) dxg[xo[k] + j] = xt - x0[k];
                            const double e = (double)xt - (double)p[k].a;
                            acc[k][1] += e * e;
                        }
                    }
            }
            __syncthreads();
            // ---- dual phase
            for (int r = 0, sl = warp; sl < nrs; ++r, sl = snake_slice(r, warp, nwarps)) {
                const int i = (sl << 5) + lane;
                const bool valid = i < m;
                RowP<MT> p[2];
#pragma unroll
                for (int k = 0; k < 2; ++k)
                    if (valid && live[k]) p[k] = rowp[yo[k] + i];
                const int2 tb = tab[ncs + sl];
                const int p0 = tb.x, len = tb.y;
                MT s[2] = {(MT)0, (MT)0};
                if (len <= kLongSlice) {
                    if (both)
                        ell_dot2<MT, W>(rev + p0 + W * lane, a.r_eidx + p0 + W * lane, len, xhb[0], xhb[1], s[0], s[1]);
                    else {
                        const MT t = ell_dot<MT, W>(rev + p0 + W * lane, a.r_eidx + p0 + W * lane, len, xh_solo);
                        s[0] = solo1 ? (MT)0 : t;
                        s[1] = solo1 ? t : (MT)0;
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        if (live[k])
                            s[k] = long_slice_dot<MT>(sv, a.rowptr, a.colidx, ro + (sl << 5), min(32, m - (sl << 5)),
                                                      co, xhb[k], lane);
                }
#pragma unroll
                for (int k = 0; k < 2; ++k)
                    if (valid && live[k]) {
                        const MT y0 = ysb[k][i];
                        MT yt = y0 + sigma[k] * (s[k] - p[k].b);
                        if (yt < p[k].lo) yt = p[k].lo;  // NaN stays NaN
                        ysb[k][i] = wk[k] * (one_rho * yt - rho * y0) + wa[k] * p[k].a;
                        if (stats[k]) {
                            const double d = (double)y0 - (double)yt;
                            acc[k][2] += d * d;
                        }
                        if (check[k]) {
                            ytg[yo[k] + i] = yt;
                            if (rays) {
                                MT d = yt - y0;
                                if (p[k].lo != (MT)(-INFINITY) && d < (MT)0) d = (MT)0;
                                dyg[yo[k] + i] = d;
                            }
                            const double e = (double)yt - (double)p[k].a;
                            acc[k][3] += e * e;
                        }
                    }
            }
#pragma unroll
            for (int k = 0; k < 2; ++k)
                if (live[k]) {
                    kk[k] += 1;
                    total[k] += 1;
                }
            if (!stats[0] && !stats[1]) {
                __syncthreads();
                continue;
            }
            // ---- per instance: restart reference residual, or the check and its decisions
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                if (!stats[k]) continue;
                block_sums<4>(acc[k], red);
                const bool was_first = first[k];
                first[k] = false;
                if (!check[k]) {
                    if (tid == 0) {
                        sc[k].r0 = sqrt(om[k] * acc[k][0] + acc[k][2] / om[k]);
                        sc[k].rprev = sc[k].r0;
                    }
                    __syncthreads();
                    continue;
                }
                double r_now = 0, dxa = 0, dya = 0;
                if (tid == 0) {
                    r_now = sqrt(om[k] * acc[k][0] + acc[k][2] / om[k]);
                    if (was_first) {
                        sc[k].r0 = r_now;
                        sc[k].rprev = r_now;
                    }
                    dxa = sqrt(acc[k][1]);
                    dya = sqrt(acc[k][3]);
                }
                __syncthreads();
                check_instance<MT, W>(a, inst[k], m, n, ro, co, xo[k], yo[k], total[k], kk[k], om[k], r_now, dxa,
                                      dya, sc[k], s_flags[k], red, tab, xhb[k]);
                __syncthreads();
                live[k] = s_flags[k][0] == 0;
                om[k] = sc[k].omega;
                if (s_flags[k][1]) {
                    kk[k] = 0;
                    first[k] = true;
                    restart_instance<MT>(a, m, n, ro, co, xo[k], yo[k], ysb[k]);
                }
                __syncthreads();
            }
        }
        // store the dual iterates and the control blocks
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (k == 0 || has2)
                for (int i = tid; i < m; i += nt) yg[yo[k] + i] = ysb[k][i];
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (tid == k && (k == 0 || has2)) {
                sc[k].k = kk[k];
                sc[k].total = total[k];
                sc[k].first = first[k] ? 1 : 0;
                a.ictrl[inst[k]] = sc[k];
            }
        __syncthreads();
    }
}

template <typename MT, int W>
__global__ void __launch_bounds__(512, 1) k_batch_pair(const __grid_constant__ BArgs a, int chunk) {
    batch_pair_body<MT, W>(a, chunk);
}

// Order-preserving compaction of the active list (one CTA).
__global__ void k_batch_compact(const InstCtrl* __restrict__ ictrl, const int32_t* __restrict__ in,
                                int32_t* __restrict__ out, int32_t* counters) {
    typedef cub::BlockScan<int, 1024> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int base;
    const int count = counters[1];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (int start = 0; start < count; start += 1024) {
        int idx = start + threadIdx.x;
        int keep = (idx < count && !ictrl[in[idx]].done) ? 1 : 0;
        int pos, tot;
        Scan(tmp).ExclusiveSum(keep, pos, tot);
        if (keep) out[base + pos] = in[idx];
        __syncthreads();
        if (threadIdx.x == 0) base += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        counters[1] = base;
        counters[0] = 0;
    }
}

// ------------------------------------------------------------------ setup kernels (CTA per matrix, FP64)
__global__ void k_batch_scaling(int nmat, const int32_t* __restrict__ mat_m, const int32_t* __restrict__ mat_n,
                                const int64_t* __restrict__ row_off, const int64_t* __restrict__ col_off,
                                const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                                const double* __restrict__ vals, const int32_t* __restrict__ t_rowptr,
                                const int32_t* __restrict__ t_colidx, const double* __restrict__ t_vals,
                                int ruiz_iters, double* __restrict__ dr, double* __restrict__ dc,
                                double* __restrict__ tmp_r, double* __restrict__ tmp_c) {
    for (int k = blockIdx.x; k < nmat; k += gridDim.x) {
        const int m = mat_m[k], n = mat_n[k];
        const int64_t ro = row_off[k], co = col_off[k];
        for (int i = threadIdx.x; i < m; i += blockDim.x) dr[ro + i] = 1.0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) dc[co + j] = 1.0;
        __syncthreads();
        for (int pass = 0; pass <= ruiz_iters; ++pass) {
            const bool pc = pass == ruiz_iters;  // last pass: Pock-Chambolle sums
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                double acc = 0.0, di = dr[ro + i];
                for (int e = rowptr[ro + i]; e < rowptr[ro + i + 1]; ++e) {
                    double v = fabs(vals[e]) * di * dc[colidx[e]];
                    acc = pc ? acc + v : fmax(acc, v);
                }
                tmp_r[ro + i] = acc;
            }
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double acc = 0.0, dj = dc[co + j];
                for (int e = t_rowptr[co + j]; e < t_rowptr[co + j + 1]; ++e) {
                    double v = fabs(t_vals[e]) * dj * dr[t_colidx[e]];
                    acc = pc ? acc + v : fmax(acc, v);
                }
                tmp_c[co + j] = acc;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < m; i += blockDim.x)
                if (tmp_r[ro + i] > 0.0) dr[ro + i] /= sqrt(tmp_r[ro + i]);
            for (int j = threadIdx.x; j < n; j += blockDim.x)
                if (tmp_c[co + j] > 0.0) dc[co + j] /= sqrt(tmp_c[co + j]);
            __syncthreads();
        }
    }
}

__global__ void k_batch_scale_vals(int64_t tot_m, int64_t tot_n, const int32_t* __restrict__ rowptr,
                                   const int32_t* __restrict__ colidx, const double* __restrict__ vals,
                                   const int32_t* __restrict__ t_rowptr, const int32_t* __restrict__ t_colidx,
                                   const double* __restrict__ t_vals, const double* __restrict__ dr,
                                   const double* __restrict__ dc, double* sv64, float* sv32, double* stv64,
                                   float* stv32) {
    int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, st = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = tid; i < tot_m; i += st) {
        double di = dr[i];
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            double v = vals[e] * di * dc[colidx[e]];
            sv64[e] = v;
            sv32[e] = (float)v;
        }
    }
    for (int64_t j = tid; j < tot_n; j += st) {
        double dj = dc[j];
        for (int e = t_rowptr[j]; e < t_rowptr[j + 1]; ++e) {
            double v = t_vals[e] * dj * dr[t_colidx[e]];
            stv64[e] = v;
            stv32[e] = (float)v;
        }
    }
}

// sigma_max(A_s)^2 per matrix by power iteration (CTA per matrix, stops at rel change 1e-7)
__global__ void k_batch_power(int nmat, const int32_t* __restrict__ mat_m, const int32_t* __restrict__ mat_n,
                              const int64_t* __restrict__ row_off, const int64_t* __restrict__ col_off,
                              const int32_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                              const double* __restrict__ sv64, const int32_t* __restrict__ t_rowptr,
                              const int32_t* __restrict__ t_colidx, const double* __restrict__ stv64, double* pv,
                              double* pu, double safety, double* __restrict__ eta_out) {
    __shared__ double red[32];
    __shared__ double s_norm, s_prev;
    __shared__ int s_stop;
    for (int k = blockIdx.x; k < nmat; k += gridDim.x) {
        const int m = mat_m[k], n = mat_n[k];
        const int64_t ro = row_off[k], co = col_off[k];
        double part = 0.0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            unsigned long long z = (unsigned long long)j * 0x9E3779B97F4A7C15ull + 0x1234567ull;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            double v = 0.5 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
            pv[co + j] = v;
            part += v * v;
        }
        double vv[1] = {part};
        block_sums<1>(vv, red);
        if (threadIdx.x == 0) {
            s_norm = sqrt(vv[0]);
            s_prev = 0.0;
            s_stop = 0;
        }
        __syncthreads();
        for (int t = 0; t < 1000 && !s_stop; ++t) {
            const double inv = 1.0 / s_norm;
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                double s = 0.0;
                for (int e = rowptr[ro + i]; e < rowptr[ro + i + 1]; ++e) s += sv64[e] * pv[colidx[e]];
                pu[ro + i] = s * inv;
            }
            __syncthreads();
            double p2 = 0.0;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double s = 0.0;
                for (int e = t_rowptr[co + j]; e < t_rowptr[co + j + 1]; ++e) s += stv64[e] * pu[t_colidx[e]];
                pv[co + j] = s;
                p2 += s * s;
            }
            double w[1] = {p2};
            block_sums<1>(w, red);
            if (threadIdx.x == 0) {
                double nn = sqrt(w[0]);
                if (nn <= 0.0 || fabs(nn - s_prev) <= 1e-7 * nn) s_stop = 1;
                s_prev = nn;
                s_norm = nn > 0.0 ? nn : 1.0;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double sig = sqrt(fmax(s_prev, 0.0));
            eta_out[k] = sig > 0.0 ? safety / sig : 1.0;
        }
        __syncthreads();
    }
}

// SELL-32 copy of one orientation, CTA per matrix: every lane slot of every slice
// (rows past the matrix end and entries past a row's end are zero padding with
// local index 0), in the W = 1 or W = 2 (pairs) order of ell_dot.  ptr / idx / v64 /
// v32 are the CSR of that orientation in global numbering; `other_off` localises its
// indices.
__global__ void k_fill_ell(int W, int nmat, const int32_t* __restrict__ dim, const int64_t* __restrict__ off,
                           const int64_t* __restrict__ other_off, const int64_t* __restrict__ s_off,
                           const int64_t* __restrict__ sptr, const int32_t* __restrict__ ptr,
                           const int32_t* __restrict__ idx, const double* __restrict__ v64,
                           const float* __restrict__ v32, uint16_t* __restrict__ eidx, double* __restrict__ ev64,
                           float* __restrict__ ev32) {
    for (int k = blockIdx.x; k < nmat; k += gridDim.x) {
        const int d = dim[k];
        const int padded = (d + 31) & ~31;
        const int64_t base = off[k], ob = other_off[k];
        const int64_t* sp = sptr + s_off[k];
        for (int li = threadIdx.x; li < padded; li += blockDim.x) {
            const int s = li >> 5, lane = li & 31;
            const int64_t p0 = sp[s];
            const int len = (int)((sp[s + 1] - p0) >> 5);
            int e = 0, e1 = 0;
            if (li < d) {
                e = ptr[base + li];
                e1 = ptr[base + li + 1];
            }
            for (int q = 0; q < len; ++q) {
                const int64_t pos = W == 1 ? p0 + 32 * (int64_t)q + lane : p0 + 64 * (int64_t)(q >> 1) + 2 * lane + (q & 1);
                if (e + q < e1) {
                    eidx[pos] = (uint16_t)(idx[e + q] - ob);
                    ev64[pos] = v64[e + q];
                    ev32[pos] = v32[e + q];
                } else {
                    eidx[pos] = 0;
                    ev64[pos] = 0.0;
                    ev32[pos] = 0.0f;
                }
            }
        }
    }
}

// Per-instance b, c, l, u, row kinds from external to internal order (CTA per instance).
__global__ void k_permute_inst(int count, const int32_t* __restrict__ inst_mat, const int32_t* __restrict__ mat_m,
                               const int32_t* __restrict__ mat_n, const int64_t* __restrict__ row_off,
                               const int64_t* __restrict__ col_off, const int64_t* __restrict__ x_off,
                               const int64_t* __restrict__ y_off, const int32_t* __restrict__ r_ext,
                               const int32_t* __restrict__ c_ext, const double* __restrict__ sb,
                               const double* __restrict__ sc, const double* __restrict__ sl,
                               const double* __restrict__ su, const uint8_t* __restrict__ seq, double* __restrict__ b,
                               double* __restrict__ c, double* __restrict__ lb, double* __restrict__ ub,
                               uint8_t* __restrict__ is_eq) {
    for (int inst = blockIdx.x; inst < count; inst += gridDim.x) {
        const int k = inst_mat[inst];
        const int m = mat_m[k], n = mat_n[k];
        const int64_t ro = row_off[k], co = col_off[k], xo = x_off[inst], yo = y_off[inst];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int64_t src = xo + c_ext[co + j];
            c[xo + j] = sc[src];
            lb[xo + j] = sl[src];
            ub[xo + j] = su[src];
        }
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const int64_t src = yo + r_ext[ro + i];
            b[yo + i] = sb[src];
            is_eq[yo + i] = seq[src];
        }
    }
}

// Per-instance norms, initial point, packed records and control block (CTA per
// instance; all `count` instances, or those named by `list`).  Warm starts arrive
// in external order.  With re-centring the initial
// point (warm start, else the bound projection of 0) becomes the first FP64
// centre and the iterates start at 0.
template <typename MT>
__global__ void k_batch_init(BArgs a, int count, const int32_t* __restrict__ list, const double* __restrict__ x0,
                             const double* __restrict__ y0, const double* __restrict__ omega0,
                             const long long* __restrict__ base0) {
    __shared__ double red[32 * 4];
    ColP<MT>* colp = (ColP<MT>*)a.colp;
    RowP<MT>* rowp = (RowP<MT>*)a.rowp;
    MT *xg = (MT*)a.x, *xtg = (MT*)a.xt, *yg = (MT*)a.y, *ytg = (MT*)a.yt;
    for (int q = blockIdx.x; q < count; q += gridDim.x) {
        const int inst = list ? list[q] : q;
        const int k = a.inst_mat[inst];
        const int m = a.mat_m[k], n = a.mat_n[k];
        const int64_t ro = a.mat_row_off[k], co = a.mat_col_off[k], xo = a.x_off[inst], yo = a.y_off[inst];
        double acc[4] = {0, 0, 0, 0};  // ||b||^2, ||c||^2, ||b_s||^2, ||c_s||^2
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double d = a.dc[co + j];
            const double cj = a.c[xo + j], lj = a.lb[xo + j], uj = a.ub[xo + j];
            const double v = clampT(x0 ? x0[xo + a.c_ext[co + j]] : 0.0, lj, uj);
            if (a.recenter) {
                a.xbar[xo + j] = v;
                xg[xo + j] = (MT)0;
                xtg[xo + j] = (MT)0;
            } else {
                const MT vs = (MT)(v / d);
                xg[xo + j] = vs;
                xtg[xo + j] = vs;
                ColP<MT> p;
                p.c = (MT)(cj * d);
                p.l = (MT)(lj / d);
                p.u = (MT)(uj / d);
                p.a = vs;
                colp[xo + j] = p;
            }
            acc[1] += cj * cj;
            acc[3] += (cj * d) * (cj * d);
        }
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const double d = a.dr[ro + i];
            const double bi = a.b[yo + i];
            const bool eq = a.is_eq[yo + i] != 0;
            double v = y0 ? y0[yo + a.r_ext[ro + i]] : 0.0;
            if (!eq && v < 0.0) v = 0.0;
            if (a.recenter) {
                a.ybar[yo + i] = v;
                yg[yo + i] = (MT)0;
                ytg[yo + i] = (MT)0;
            } else {
                const MT vs = (MT)(v / d);
                yg[yo + i] = vs;
                ytg[yo + i] = vs;
                RowP<MT> r;
                r.b = (MT)(bi * d);
                r.lo = eq ? (MT)(-INFINITY) : (MT)0;
                r.a = vs;
                r.pad = (MT)0;
                rowp[yo + i] = r;
            }
            acc[0] += bi * bi;
            acc[2] += (bi * d) * (bi * d);
        }
        block_sums<4>(acc, red);
        if (threadIdx.x == 0) {
            a.bnorm[inst] = sqrt(acc[0]);
            a.cnorm[inst] = sqrt(acc[1]);
            const double bn = sqrt(acc[2]), cn = sqrt(acc[3]);
            InstCtrl s;
            memset(&s, 0, sizeof(s));
            s.omega = (omega0 && omega0[inst] > 0.0) ? omega0[inst] : ((bn > 1e-10 && cn > 1e-10) ? cn / bn : 1.0);
            s.first = 1;
            s.base = base0 ? base0[q] : 0;
            s.status = B2P_STATUS_MAX_ITERATIONS;
            a.ictrl[inst] = s;
        }
        if (a.recenter) {
            __syncthreads();  // the centre of this instance is complete
            rebuild_shifted<MT>(a, m, n, ro, co, xo, yo);
        }
        __syncthreads();
    }
}

// Answers in the original space and external order: x = xbar + dc * xt, y = ybar + dr * yt.
template <typename T>
__global__ void k_batch_unscale(BArgs a, int count, const double* __restrict__ xbar, const double* __restrict__ ybar,
                                double* __restrict__ xo_, double* __restrict__ yo_) {
    const T* xt = (const T*)a.xt;
    const T* yt = (const T*)a.yt;
    for (int inst = blockIdx.x; inst < count; inst += gridDim.x) {
        const int k = a.inst_mat[inst];
        const int m = a.mat_m[k], n = a.mat_n[k];
        const int64_t ro = a.mat_row_off[k], co = a.mat_col_off[k], xo = a.x_off[inst], yo = a.y_off[inst];
        for (int j = threadIdx.x; j < n; j += blockDim.x)
            xo_[xo + a.c_ext[co + j]] = (xbar ? xbar[xo + j] : 0.0) + a.dc[co + j] * (double)xt[xo + j];
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            yo_[yo + a.r_ext[ro + i]] = (ybar ? ybar[yo + i] : 0.0) + a.dr[ro + i] * (double)yt[yo + i];
    }
}

// ------------------------------------------------------------------ host side
struct TuneCfg {
    int threads, chunk, w;  // CTA size, iterations per chunk launch, SELL entries per lane load (1 or 2)
    int ni;                 // instances per CTA: 1, or 2 (paired form, batches of one shared matrix)
};

// Candidate shapes of the autotuner: CTA sizes, SELL entry orders and instances per CTA
// (2 only when every instance shares one matrix).  B2P_BATCH_SHAPE="threads,w,ni" pins
// all three (the chunk length is still tuned); a pinned pair on a batch of several
// matrices falls back to one instance per CTA.
struct ShapeChoices {
    std::vector<int> threads{128, 256, 512}, w{1, 2}, ni{1, 2};
};

ShapeChoices shape_choices(BatchWork* w) {
    ShapeChoices c;
    const bool can_pair = w->nmat == 1 && w->count > 1;
    if (!can_pair) c.ni = {1};
    const char* e = std::getenv("B2P_BATCH_SHAPE");
    int th = 0, ww = 0, ni = 0;
    if (e && std::sscanf(e, "%d,%d,%d", &th, &ww, &ni) == 3 && (th == 128 || th == 256 || th == 512) &&
        (ww == 1 || ww == 2) && (ni == 1 || ni == 2)) {
        c.threads = {th};
        c.w = {ww};
        c.ni = {can_pair ? ni : 1};
    }
    return c;
}

std::string cache_path() {
    const char* p = std::getenv("B2P_AUTOTUNE_CACHE");
    if (p && *p) return p;
    const char* h = std::getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/b2p_autotune.txt";
}

std::string batch_key(BatchWork* w, int precision) {
    // signature: kernel version, precision, size classes of the batch
    double mean_m = (double)w->inst_m / w->count, mean_n = (double)w->inst_n / w->count;
    double nnz_col = (double)w->nnz / std::max<int64_t>(w->tot_n, 1);
    std::ostringstream os;
    const char* f = std::getenv("B2P_BATCH_SHAPE");
    os << "batch6" << (f && *f ? std::string("_s") + f : std::string()) << "_p" << precision << "_c" << (int)std::log2(std::max(1, w->count)) << "_m"
       << (int)std::log2(mean_m + 1) << "_n" << (int)std::log2(mean_n + 1) << "_k" << (int)std::lround(nnz_col) << "_M"
       << w->max_m << "_N" << w->max_n << "_shared" << (w->nmat == 1 && w->count > 1);
    return os.str();
}

bool cache_lookup(const std::string& key, TuneCfg* out) {
    std::ifstream f(cache_path());
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string k;
        TuneCfg c;
        if (!(is >> k) || k != key) continue;
        if (is >> c.threads >> c.chunk >> c.w >> c.ni) {
            *out = c;
            return true;
        }
    }
    return false;
}

void cache_store(const std::string& key, const TuneCfg& c) {
    std::string p = cache_path();
    std::string dir = p.substr(0, p.find_last_of('/'));
    if (!dir.empty()) {
        std::string cmd = "mkdir -p '" + dir + "'";
        if (std::system(cmd.c_str()) != 0) return;
    }
    std::ofstream f(p, std::ios::app);
    f << key << " " << c.threads << " " << c.chunk << " " << c.w << " " << c.ni << "\n";
}

template <typename MT>
BArgs make_args(BatchWork* w, const b2p_params* p, const int32_t* active) {
    const bool f64 = sizeof(MT) == 8;
    BArgs a;
    a.rowptr = w->rowptr.p;
    a.colidx = w->colidx.p;
    a.t_rowptr = w->t_rowptr.p;
    a.t_colidx = w->t_colidx.p;
    a.sv64 = w->sv64.p;
    a.stv64 = w->stv64.p;
    a.dr = w->dr.p;
    a.dc = w->dc.p;
    a.mat_eta = w->mat_eta.p;
    a.sv = f64 ? (const void*)w->sv64.p : (const void*)w->sv32.p;
    a.stv = f64 ? (const void*)w->stv64.p : (const void*)w->stv32.p;
    a.mat_m = w->mat_m.p;
    a.mat_n = w->mat_n.p;
    a.mat_row_off = w->mat_row_off.p;
    a.mat_col_off = w->mat_col_off.p;
    a.r_sptr = w->r_sptr.p;
    a.c_sptr = w->c_sptr.p;
    a.mat_rs_off = w->mat_rs_off.p;
    a.mat_cs_off = w->mat_cs_off.p;
    a.r_eidx = w->r_eidx.p;
    a.c_eidx = w->c_eidx.p;
    a.r_ev = f64 ? (const void*)w->r_ev64.p : (const void*)w->r_ev32.p;
    a.c_ev = f64 ? (const void*)w->c_ev64.p : (const void*)w->c_ev32.p;
    a.r_ev64 = w->r_ev64.p;
    a.c_ev64 = w->c_ev64.p;
    a.r_ext = w->r_ext.p;
    a.c_ext = w->c_ext.p;
    a.inst_mat = w->inst_mat.p;
    a.x_off = w->x_off.p;
    a.y_off = w->y_off.p;
    a.b = w->b.p;
    a.c = w->c.p;
    a.lb = w->lb.p;
    a.ub = w->ub.p;
    a.bnorm = w->bnorm.p;
    a.cnorm = w->cnorm.p;
    a.is_eq = w->is_eq.p;
    a.colp = w->colp.p;
    a.rowp = w->rowp.p;
    a.x = w->x.p;
    a.xt = w->xt.p;
    a.y = w->y.p;
    a.yt = w->yt.p;
    a.dx = w->dx.p;
    a.dy = w->dy.p;
    a.ictrl = w->ictrl.p;
    a.active = active;
    a.counters = w->counters.p;
    a.eps = p->eps_rel_kkt;
    a.beta_s = p->restart_sufficient;
    a.beta_n = p->restart_necessary;
    a.beta_a = p->restart_artificial;
    a.rho = p->reflection;
    a.eps_obj = p->eps_objective;
    a.eps_inf = (w->dx.p && w->dy.p) ? p->eps_infeasible : 0.0;
    a.max_iter = p->max_iterations;
    a.K = p->check_every;
    a.recenter = w->recenter ? 1 : 0;
    a.vals = w->vals.p;
    a.t_vals = w->t_vals.p;
    a.xbar = w->xbar.p;
    a.ybar = w->ybar.p;
    a.axbar = w->axbar.p;
    a.atybar = w->atybar.p;
    return a;
}

// dynamic shared memory of one CTA: y and xh (MT) of the largest instance, or of two
// instances of the shared matrix in the paired form
size_t smem_bytes(BatchWork* w, size_t mt_size, int ni = 1) {
    const size_t tab = sizeof(int2) * slice_tab_len((w->max_m + 31) >> 5, (w->max_n + 31) >> 5);
    const size_t m4 = (size_t)((w->max_m + 3) & ~3), n4 = (size_t)((w->max_n + 3) & ~3);
    return tab + mt_size * ni * (m4 + std::max(n4, m4)) + 16;  // y, then xh (which also stages y at checks)
}

// The chunk kernel of a tuned shape.
template <typename MT>
void (*chunk_kernel(int w, int ni))(const BArgs, int) {
    if (ni == 2) return w == 2 ? k_batch_pair<MT, 2> : k_batch_pair<MT, 1>;
    return w == 2 ? k_batch_chunk<MT, 2> : k_batch_chunk<MT, 1>;
}

template <typename MT>
int init_instances(Ctx* ctx, BatchWork* w, const b2p_params* p, const double* x0_dev, const double* y0_dev,
                   const double* om_dev, const int32_t* list_dev = nullptr, int list_count = 0,
                   const long long* base_dev = nullptr) {
    const int cnt = list_dev ? list_count : w->count;
    int grid = std::min(cnt, ctx->sm_count * 8);
    BArgs a = make_args<MT>(w, p, w->active.p);
    k_batch_init<MT><<<grid, 256, 0, ctx->stream>>>(a, cnt, list_dev, x0_dev, y0_dev, om_dev, base_dev);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    return B2P_OK;
}

// Rewrites both SELL copies in entry order W (1 or 2); the slice pointers (even lengths)
// serve both orders.
int refill_ell(Ctx* ctx, BatchWork* w, int W) {
    if (w->ell_w == W) return B2P_OK;
    cudaStream_t s = ctx->stream;
    const unsigned gmat = (unsigned)std::min(w->nmat, ctx->sm_count * 8);
    k_fill_ell<<<gmat, 256, 0, s>>>(W, w->nmat, w->mat_m.p, w->mat_row_off.p, w->mat_col_off.p, w->mat_rs_off.p,
                                     w->r_sptr.p, w->rowptr.p, w->colidx.p, w->sv64.p, w->sv32.p, w->r_eidx.p,
                                     w->r_ev64.p, w->r_ev32.p);
    k_fill_ell<<<gmat, 256, 0, s>>>(W, w->nmat, w->mat_n.p, w->mat_col_off.p, w->mat_row_off.p, w->mat_cs_off.p,
                                     w->c_sptr.p, w->t_rowptr.p, w->t_colidx.p, w->stv64.p, w->stv32.p, w->c_eidx.p,
                                     w->c_ev64.p, w->c_ev32.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 2;
    w->ell_w = W;
    return B2P_OK;
}

// Times each shape on a size-stratified sample of the batch (no termination, 4a
// iterations -- long enough that the restart checks weigh as in a real solve -- no
// re-centring), then the chunk length: with the chosen shape, launches of a and 4a
// iterations give the per-iteration cost p and the fixed cost o of a chunk (launch, loading and storing every instance's state, plus the
// compaction that follows); the chunk is the shortest power of two from 256 to 8192
// whose fixed cost is at most 2 % of its iterations -- shorter chunks drop finished
// instances sooner, so the tail of an uneven batch is cut finer.  Each block size is
// tried with both SELL entry orders (one entry or a pair per lane load) and, when every
// instance shares one matrix, in the single and the paired form (two instances per
// CTA).  Instance state is re-initialised afterwards by the caller.
template <typename MT>
int autotune(Ctx* ctx, BatchWork* w, const b2p_params* p, TuneCfg* best) {
    std::string key = batch_key(w, sizeof(MT) == 8 ? 0 : 1);
    if (cache_lookup(key, best)) return B2P_OK;
    cudaStream_t s = ctx->stream;
    int sample = std::min(w->count, ctx->sm_count * 4);
    std::vector<int32_t> ids(sample);
    for (int i = 0; i < sample; ++i) ids[i] = w->order[(int64_t)i * w->count / sample];
    DBuf<int32_t> dids;
    B2P_CUDA(ctx, dids.reserve(sample));
    B2P_CUDA(ctx, cudaMemcpyAsync(dids.p, ids.data(), sizeof(int32_t) * sample, cudaMemcpyHostToDevice, s));
    b2p_params tp = *p;
    tp.max_iterations = 1LL << 40;
    tp.eps_rel_kkt = 0.0;  // never terminates inside the trial
    tp.eps_infeasible = 0.0;
    const int trial_iters = 128;
    float best_ms = 1e30f;
    *best = {256, 2048, 1, 1};
    int max_smem = 0;
    B2P_CUDA(ctx, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    // one trial launch of `iters` iterations over the sample with `th` threads, entry order W
    // and ni instances per CTA (ms; < 0: the shape does not fit)
    auto trial = [&](int th, int W, int ni, int iters, float* ms) -> int {
        *ms = -1.0f;
        auto fn = chunk_kernel<MT>(W, ni);
        const size_t sm = smem_bytes(w, sizeof(MT), ni);
        if (sm > (size_t)max_smem) return B2P_OK;
        B2P_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int st = refill_ell(ctx, w, W);
        if (st) return st;
        st = init_instances<MT>(ctx, w, &tp, nullptr, nullptr, nullptr);
        if (st) return st;
        int32_t cnt[2] = {0, sample};
        B2P_CUDA(ctx, cudaMemcpyAsync(w->counters.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s));
        BArgs a = make_args<MT>(w, &tp, dids.p);
        int per_sm = 0;
        B2P_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, th, sm));
        if (per_sm < 1) return B2P_OK;
        int grid = std::min((sample + ni - 1) / ni, ctx->sm_count * per_sm);
        cudaEventRecord(ctx->ev0, s);
        fn<<<grid, th, sm, s>>>(a, iters);
        k_batch_compact<<<1, 1024, 0, s>>>(w->ictrl.p, dids.p, w->active2.p, w->counters.p);
        cudaEventRecord(ctx->ev1, s);
        B2P_LAUNCH(ctx);
        B2P_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
        ctx->launches += 2;
        cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1);
        return B2P_OK;
    };
    const ShapeChoices choices = shape_choices(w);
    for (int ni : choices.ni)
        for (int W : choices.w)
            for (int th : choices.threads) {
                float ms = 0.0f;
                int st = trial(th, W, ni, 4 * trial_iters, &ms);
                if (st) return st;
                if (ms >= 0.0f && ms < best_ms) {
                    best_ms = ms;
                    best->threads = th;
                    best->w = W;
                    best->ni = ni;
                }
            }
    if (best_ms >= 1e30f) {
        ctx->err = "batch: no chunk-kernel shape fits this batch";
        return B2P_INVALID_ARGUMENT;
    }
    float t1 = 0.0f;
    int st = trial(best->threads, best->w, best->ni, trial_iters, &t1);
    if (st) return st;
    const double per_iter = std::max(1e-9, (double)(best_ms - t1) / (3.0 * trial_iters));
    const double fixed = std::max(0.0, (double)t1 - trial_iters * per_iter);
    int chunk = 256;
    while (chunk < 8192 && fixed > 0.02 * chunk * per_iter) chunk *= 2;
    best->chunk = chunk;
    cache_store(key, *best);
    return B2P_OK;
}

template <typename MT>
int batch_run(Ctx* ctx, BatchWork* w, const b2p_params* p, const double* x0_dev, const double* y0_dev,
              const double* om_dev, const std::vector<int32_t>* subset, bool* timed_out_out, float* kms_out,
              TuneCfg* cfg_out, const std::vector<long long>* base = nullptr) {
    cudaStream_t s = ctx->stream;
    double t_start = now_ms();
    const int64_t IN = w->inst_n, IM = w->inst_m;
    const int prec = sizeof(MT) == 8 ? 0 : 1;
    {
        // y and xh of the largest instance must fit one CTA's shared memory
        int max_smem = 0;
        B2P_CUDA(ctx, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
        const size_t need = smem_bytes(w, sizeof(MT));
        if (need > (size_t)max_smem) {
            ctx->err = "batch instance too large for one CTA's shared memory: needs " + std::to_string(need) +
                       " bytes (" + std::to_string(w->max_m) + " rows + " + std::to_string(w->max_n) +
                       " columns), the device allows " + std::to_string(max_smem) +
                       "; solve it with b2p_solve";
            return B2P_INVALID_ARGUMENT;
        }
    }
    w->recenter = false;  // autotune trials run without re-centring
    TuneCfg cfg = {256, 2048, 1, 1};
    if (w->tuned_threads[prec] > 0) {
        cfg.threads = w->tuned_threads[prec];
        cfg.chunk = w->tuned_chunk[prec];
        cfg.w = w->tuned_w[prec];
        cfg.ni = w->tuned_ni[prec];
    } else {
        if (subset) {
            ctx->err = "subset solve before a full solve of this precision";
            return B2P_INVALID_ARGUMENT;
        }
        int st = autotune<MT>(ctx, w, p, &cfg);
        if (st) return st;
        w->tuned_threads[prec] = cfg.threads;
        w->tuned_chunk[prec] = cfg.chunk;
        w->tuned_w[prec] = cfg.w;
        w->tuned_ni[prec] = cfg.ni;
    }
    {
        int st = refill_ell(ctx, w, cfg.w);
        if (st) return st;
    }
    // displacement buffers of the infeasibility certificates (sized for FP64, read as MT)
    if (p->eps_infeasible > 0.0) {
        B2P_CUDA(ctx, w->dx.reserve(IN));
        B2P_CUDA(ctx, w->dy.reserve(IM));
    }
    // re-centring: on by default for the mixed engine (refinement_rounds < 0), forced by > 0
    w->recenter = p->refinement_rounds > 0 || (p->refinement_rounds < 0 && sizeof(MT) == 4);
    if (w->recenter) {
        for (auto* b : {&w->xbar, &w->atybar}) B2P_CUDA(ctx, b->reserve(IN));
        for (auto* b : {&w->ybar, &w->axbar}) B2P_CUDA(ctx, b->reserve(IM));
    }
    // instances to run, longest first
    std::vector<int32_t> act;
    if (subset) {
        std::vector<uint8_t> in_set(w->count, 0);
        for (int32_t i : *subset) in_set[i] = 1;
        for (int32_t i : w->order)
            if (in_set[i]) act.push_back(i);
        if (act.empty()) {
            if (timed_out_out) *timed_out_out = false;
            if (kms_out) *kms_out = 0.0f;
            if (cfg_out) *cfg_out = cfg;
            return B2P_OK;
        }
        B2P_CUDA(ctx, w->list.reserve(act.size()));
        B2P_CUDA(ctx, cudaMemcpyAsync(w->list.p, act.data(), sizeof(int32_t) * act.size(), cudaMemcpyHostToDevice, s));
        DBuf<long long> dbase;
        if (base) {  // per listed instance, in list order
            std::vector<long long> b(act.size());
            for (size_t q = 0; q < act.size(); ++q) b[q] = (*base)[act[q]];
            B2P_CUDA(ctx, dbase.reserve(act.size()));
            B2P_CUDA(ctx, cudaMemcpyAsync(dbase.p, b.data(), sizeof(long long) * b.size(), cudaMemcpyHostToDevice, s));
        }
        int st = init_instances<MT>(ctx, w, p, x0_dev, y0_dev, om_dev, w->list.p, (int)act.size(),
                                    base ? dbase.p : nullptr);
        if (st) return st;
        B2P_CUDA(ctx, cudaStreamSynchronize(s));  // dbase is released at scope end
    } else {
        act = w->order;
        int st = init_instances<MT>(ctx, w, p, x0_dev, y0_dev, om_dev);
        if (st) return st;
    }
    const int n_act = (int)act.size();
    B2P_CUDA(ctx, cudaMemcpyAsync(w->active.p, act.data(), sizeof(int32_t) * n_act, cudaMemcpyHostToDevice, s));
    int32_t cnt[2] = {0, n_act};
    B2P_CUDA(ctx, cudaMemcpyAsync(w->counters.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s));
    const size_t sm_main = smem_bytes(w, sizeof(MT), cfg.ni);
    auto fn = chunk_kernel<MT>(cfg.w, cfg.ni);
    B2P_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_main));
    int per_sm = 0;
    B2P_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, cfg.threads, sm_main));
    if (per_sm < 1) {
        ctx->err = "batch instance too large for one CTA's shared memory";
        return B2P_INVALID_ARGUMENT;
    }
    const int grid = ctx->sm_count * per_sm;
    const size_t sm = smem_bytes(w, sizeof(MT));  // the wide (single) form
    BArgs a1 = make_args<MT>(w, p, w->active.p);
    BArgs a2 = make_args<MT>(w, p, w->active2.p);
    // the wide form for the tail: 1024 threads, one CTA per SM
    auto fnw = cfg.w == 2 ? k_batch_chunk_wide<MT, 2> : k_batch_chunk_wide<MT, 1>;
    B2P_CUDA(ctx, cudaFuncSetAttribute(fnw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm_w = 0;
    B2P_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_w, fnw, 1024, sm));
    const bool have_wide = per_sm_w >= 1;
    const int grid_w = ctx->sm_count * std::max(per_sm_w, 1);
    // one graph = two chunk launches with compaction (ping-pong active lists); a second
    // graph does the same with the wide kernel.  The guard releases the graphs, their
    // executables and the pinned counter copy on every way out of this function.
    struct Owned {
        cudaGraph_t graph[2] = {nullptr, nullptr};
        cudaGraphExec_t exec[2] = {nullptr, nullptr};
        int32_t* host_cnt = nullptr;
        ~Owned() {
            for (int g = 0; g < 2; ++g) {
                if (exec[g]) cudaGraphExecDestroy(exec[g]);
                if (graph[g]) cudaGraphDestroy(graph[g]);
            }
            if (host_cnt) cudaFreeHost(host_cnt);
        }
    } own;
    cudaGraph_t& graph = own.graph[0];
    cudaGraph_t& graph_w = own.graph[1];
    cudaGraphExec_t& exec = own.exec[0];
    cudaGraphExec_t& exec_w = own.exec[1];
    for (int g = 0; g < (have_wide ? 2 : 1); ++g) {
        B2P_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (g == 0) fn<<<grid, cfg.threads, sm_main, s>>>(a1, cfg.chunk);
        else fnw<<<grid_w, 1024, sm, s>>>(a1, cfg.chunk);
        k_batch_compact<<<1, 1024, 0, s>>>(w->ictrl.p, w->active.p, w->active2.p, w->counters.p);
        if (g == 0) fn<<<grid, cfg.threads, sm_main, s>>>(a2, cfg.chunk);
        else fnw<<<grid_w, 1024, sm, s>>>(a2, cfg.chunk);
        k_batch_compact<<<1, 1024, 0, s>>>(w->ictrl.p, w->active2.p, w->active.p, w->counters.p);
        cudaGraph_t& gr = g == 0 ? graph : graph_w;
        cudaGraphExec_t& ex = g == 0 ? exec : exec_w;
        cudaError_t ce = cudaStreamEndCapture(s, &gr);
        if (ce != cudaSuccess) {
            gr = nullptr;
            ctx->err = std::string("batch graph capture: ") + cudaGetErrorString(ce);
            return B2P_EXECUTION_FAILED;
        }
        ce = cudaGraphInstantiate(&ex, gr, 0);
        if (ce != cudaSuccess) {
            ex = nullptr;
            ctx->err = std::string("batch graph instantiate: ") + cudaGetErrorString(ce);
            return B2P_EXECUTION_FAILED;
        }
    }
    int32_t*& host_cnt = own.host_cnt;
    B2P_CUDA(ctx, cudaMallocHost(&host_cnt, 2 * sizeof(int32_t)));
    const int64_t max_graphs = p->max_iterations / (2LL * cfg.chunk) + 3;
    int64_t graphs = 0;
    bool timed_out = false;
    const double tl = p->time_limit_s * 1000.0;
    cudaEventRecord(ctx->ev0, s);
    // no more than one instance per SM left: the wide form
    bool wide = have_wide && n_act <= ctx->sm_count;
    const double trace_base = subset && !w->trace_ms.empty() ? w->trace_ms.back() : 0.0;
    if (!subset) {
        w->trace_ms.clear();
        w->trace_active.clear();
    }
    const double t_loop = now_ms();
    w->trace_ms.push_back(trace_base);
    w->trace_active.push_back(n_act);
    while (graphs < max_graphs) {
        B2P_CUDA(ctx, cudaGraphLaunch(wide ? exec_w : exec, s));
        graphs++;
        B2P_CUDA(ctx, cudaMemcpyAsync(host_cnt, w->counters.p, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        w->trace_ms.push_back(trace_base + now_ms() - t_loop);
        w->trace_active.push_back(host_cnt[1]);
        if (host_cnt[1] == 0) break;
        if (have_wide && host_cnt[1] <= ctx->sm_count) wide = true;
        if (tl > 0 && now_ms() - t_start > tl) {
            timed_out = true;
            break;
        }
    }
    cudaEventRecord(ctx->ev1, s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    ctx->launches += graphs * 4;
    float kms = 0;
    cudaEventElapsedTime(&kms, ctx->ev0, ctx->ev1);
    // results of every instance: control blocks to the host, answers (original space,
    // external order) and primal weights kept on the device
    w->hc.resize(w->count);
    B2P_CUDA(ctx, cudaMemcpyAsync(w->hc.data(), w->ictrl.p, sizeof(InstCtrl) * w->count, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, w->ox.reserve(IN));
    B2P_CUDA(ctx, w->oy.reserve(IM));
    B2P_CUDA(ctx, w->oom.reserve(w->count));
    k_batch_unscale<MT><<<std::min(w->count, ctx->sm_count * 8), 256, 0, s>>>(
        a1, w->count, w->recenter ? w->xbar.p : nullptr, w->recenter ? w->ybar.p : nullptr, w->ox.p, w->oy.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    std::vector<double> om(w->count);
    for (int i = 0; i < w->count; ++i) om[i] = w->hc[i].omega;
    B2P_CUDA(ctx, cudaMemcpyAsync(w->oom.p, om.data(), sizeof(double) * w->count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    w->solved = true;
    if (timed_out_out) *timed_out_out = timed_out;
    if (kms_out) *kms_out = kms;
    if (cfg_out) *cfg_out = cfg;
    return B2P_OK;
}

// Per-instance outputs of the last solve (any pointer may be null).
int collect_outputs(Ctx* ctx, BatchWork* w, bool timed_out, int32_t* status_out, int64_t* iters_out, double* kkt_out,
                    double* omega_out, double* x_out, double* y_out, int64_t* tot_it, int64_t* maxit, int64_t* opt,
                    double* worst) {
    cudaStream_t s = ctx->stream;
    *tot_it = 0;
    *maxit = 0;
    *opt = 0;
    *worst = 0.0;
    for (int i = 0; i < w->count; ++i) {
        const InstCtrl& c = w->hc[i];
        int stt = c.done ? c.status : (timed_out ? B2P_STATUS_INTERRUPTED : B2P_STATUS_MAX_ITERATIONS);
        double kk = std::max(c.rel_p, std::max(c.rel_d, c.rel_g));
        if (status_out) status_out[i] = stt;
        if (iters_out) iters_out[i] = c.total + c.base;
        if (kkt_out) kkt_out[i] = kk;
        if (omega_out) omega_out[i] = c.omega;
        *tot_it += c.total + c.base;
        *maxit = std::max<int64_t>(*maxit, c.total + c.base);
        *opt += (stt == B2P_STATUS_OPTIMAL);
        *worst = std::max(*worst, kk);
    }
    if (x_out) B2P_CUDA(ctx, cudaMemcpyAsync(x_out, w->ox.p, sizeof(double) * w->inst_n, cudaMemcpyDeviceToHost, s));
    if (y_out) B2P_CUDA(ctx, cudaMemcpyAsync(y_out, w->oy.p, sizeof(double) * w->inst_m, cudaMemcpyDeviceToHost, s));
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    return B2P_OK;
}

void fill_summary(b2p_result* sum, int count, bool timed_out, int64_t tot_it, int64_t maxit, int64_t opt, double worst,
                  float kms, const TuneCfg& cfg) {
    if (!sum) return;
    sum->status = (opt == count) ? B2P_STATUS_OPTIMAL : (timed_out ? B2P_STATUS_INTERRUPTED : B2P_STATUS_MAX_ITERATIONS);
    sum->iterations = tot_it;  // sum over instances
    sum->restarts = maxit;     // longest instance
    sum->rel_kkt = worst;
    sum->kernel_time_ms = kms;
    sum->primal_weight = 0.0;
    sum->step_size = cfg.threads * 100000.0 + cfg.chunk;  // tuned block size * 1e5 + chunk length
    sum->used_average = 10 * cfg.ni + cfg.w;                // 10 * instances per CTA + SELL entries per lane load
}

// All instances of the batch share one shape (required by the learned warm start).
bool uniform_shape(BatchWork* w, int* n, int* m) {
    *n = w->h_mat_n[w->h_inst_mat[0]];
    *m = w->h_mat_m[w->h_inst_mat[0]];
    for (int i = 1; i < w->count; ++i)
        if (w->h_mat_n[w->h_inst_mat[i]] != *n || w->h_mat_m[w->h_inst_mat[i]] != *m) return false;
    return true;
}

}  // namespace
}  // namespace b2p

using namespace b2p;

extern "C" {

int b2p_batch_upload(void* p, int nmat, const int32_t* mat_m, const int32_t* mat_n, const int64_t* mat_nnz_off,
                     const int32_t* rowptr, const int32_t* colidx, const double* vals, int count,
                     const int32_t* inst_mat, const double* b, const double* c, const double* lb, const double* ub,
                     const uint8_t* is_eq) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (nmat <= 0 || count <= 0 || !mat_m || !mat_n || !mat_nnz_off || !rowptr || !inst_mat || !b || !c || !lb || !ub ||
        !is_eq) {
        ctx->err = "b2p_batch_upload: empty batch or null argument";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    batch_free(ctx);
    BatchWork* w = new BatchWork();
    ctx->bw = w;
    w->nmat = nmat;
    w->count = count;
    std::vector<int64_t> row_off(nmat), col_off(nmat);
    int64_t tm = 0, tn = 0;
    for (int k = 0; k < nmat; ++k) {
        if (mat_m[k] <= 0 || mat_n[k] <= 0) {
            ctx->err = "b2p_batch_upload: empty matrix";
            return B2P_INVALID_ARGUMENT;
        }
        if (mat_m[k] > 65535 || mat_n[k] > 65535) {
            ctx->err = "b2p_batch_upload: a batched instance has at most 65535 rows and columns";
            return B2P_INVALID_ARGUMENT;
        }
        row_off[k] = tm;
        col_off[k] = tn;
        tm += mat_m[k];
        tn += mat_n[k];
        w->max_m = std::max(w->max_m, mat_m[k]);
        w->max_n = std::max(w->max_n, mat_n[k]);
    }
    const int64_t nnz = mat_nnz_off[nmat];
    if (nnz > INT32_MAX || tm > INT32_MAX || tn > INT32_MAX) {
        ctx->err = "b2p_batch_upload: batch exceeds 32-bit index range";
        return B2P_INVALID_ARGUMENT;
    }
    w->tot_m = tm;
    w->tot_n = tn;
    w->nnz = nnz;
    // validate, then renumber rows and columns of each matrix by decreasing length
    // (stable) and build the internal CSR (global indices) and the SELL-32 slice
    // pointers of both orientations
    std::vector<int32_t> grp(tm + 1), gci(nnz), r_ext(tm), c_ext(tn);
    std::vector<double> gval(nnz);
    std::vector<int64_t> rs_off(nmat), cs_off(nmat), r_sptr, c_sptr;
    r_sptr.reserve(tm / 32 + 2 * nmat);
    c_sptr.reserve(tn / 32 + 2 * nmat);
    int64_t rp_base = 0, r_pad = 0, c_pad = 0, pos = 0;
    grp[0] = 0;
    std::vector<int32_t> rlen, clen, rord, cord, cinv;
    for (int k = 0; k < nmat; ++k) {
        const int32_t* rp = rowptr + rp_base;
        const int m = mat_m[k], n = mat_n[k];
        const int64_t e0 = mat_nnz_off[k], e1 = mat_nnz_off[k + 1];
        if (rp[0] != 0 || rp[m] != e1 - e0) {
            ctx->err = "b2p_batch_upload: matrix " + std::to_string(k) + " row pointers do not match its nnz";
            return B2P_INVALID_ARGUMENT;
        }
        rlen.assign(m, 0);
        clen.assign(n, 0);
        for (int i = 0; i < m; ++i) {
            if (rp[i + 1] < rp[i]) {
                ctx->err = "b2p_batch_upload: decreasing row pointer";
                return B2P_INVALID_ARGUMENT;
            }
            int prev = -1;
            for (int e = rp[i]; e < rp[i + 1]; ++e) {
                int cidx = colidx[e0 + e];
                if (cidx < 0 || cidx >= n || cidx <= prev) {
                    ctx->err = "b2p_batch_upload: matrix " + std::to_string(k) + " row " + std::to_string(i) +
                               ": column indices out of range or not strictly ascending";
                    return B2P_INVALID_ARGUMENT;
                }
                prev = cidx;
                clen[cidx]++;
            }
            rlen[i] = rp[i + 1] - rp[i];
        }
        rord.resize(m);
        cord.resize(n);
        std::iota(rord.begin(), rord.end(), 0);
        std::iota(cord.begin(), cord.end(), 0);
        std::stable_sort(rord.begin(), rord.end(), [&](int x, int y) { return rlen[x] > rlen[y]; });
        std::stable_sort(cord.begin(), cord.end(), [&](int x, int y) { return clen[x] > clen[y]; });
        cinv.resize(n);
        for (int j = 0; j < n; ++j) {
            cinv[cord[j]] = j;
            c_ext[col_off[k] + j] = cord[j];
        }
        for (int i = 0; i < m; ++i) {
            const int old = rord[i];
            r_ext[row_off[k] + i] = old;
            for (int e = rp[old]; e < rp[old + 1]; ++e) {
                gci[pos] = (int32_t)(cinv[colidx[e0 + e]] + col_off[k]);
                gval[pos] = vals[e0 + e];
                ++pos;
            }
            grp[row_off[k] + i + 1] = (int32_t)pos;
        }
        // slice pointers: matrix k owns nslices + 1 entries
        rs_off[k] = (int64_t)r_sptr.size();
        for (int s0 = 0; s0 < m; s0 += 32) {
            r_sptr.push_back(r_pad);
            r_pad += 32LL * ((rlen[rord[s0]] + 1) & ~1);  // even: both entry orders (W = 1, 2) fit
        }
        r_sptr.push_back(r_pad);
        cs_off[k] = (int64_t)c_sptr.size();
        for (int s0 = 0; s0 < n; s0 += 32) {
            c_sptr.push_back(c_pad);
            c_pad += 32LL * ((clen[cord[s0]] + 1) & ~1);
        }
        c_sptr.push_back(c_pad);
        if (r_pad > INT32_MAX || c_pad > INT32_MAX) {  // the kernels' slice tables hold 32-bit offsets
            ctx->err = "b2p_batch_upload: the batch's padded matrices exceed 2^31 entries; split the batch";
            return B2P_INVALID_ARGUMENT;
        }
        rp_base += m + 1;
    }
    w->h_mat_m.assign(mat_m, mat_m + nmat);
    w->h_mat_n.assign(mat_n, mat_n + nmat);
    // instances
    std::vector<int64_t> xoff(count), yoff(count);
    int64_t IN = 0, IM = 0;
    std::vector<int64_t> inst_nnz(count);
    for (int i = 0; i < count; ++i) {
        int k = inst_mat[i];
        if (k < 0 || k >= nmat) {
            ctx->err = "b2p_batch_upload: instance names a matrix out of range";
            return B2P_INVALID_ARGUMENT;
        }
        xoff[i] = IN;
        yoff[i] = IM;
        IN += mat_n[k];
        IM += mat_m[k];
        inst_nnz[i] = mat_nnz_off[k + 1] - mat_nnz_off[k];
    }
    w->inst_n = IN;
    w->inst_m = IM;
    for (int64_t j = 0; j < IN; ++j)
        if (std::isnan(c[j]) || std::isnan(lb[j]) || std::isnan(ub[j])) {
            ctx->err = "b2p_batch_upload: NaN in c / lb / ub";
            return B2P_INVALID_ARGUMENT;
        }
    w->h_inst_mat.assign(inst_mat, inst_mat + count);
    w->order.resize(count);
    std::iota(w->order.begin(), w->order.end(), 0);
    std::stable_sort(w->order.begin(), w->order.end(),
                     [&](int a, int b2) { return inst_nnz[a] > inst_nnz[b2]; });
    cudaStream_t s = ctx->stream;
    B2P_CUDA(ctx, w->rowptr.reserve(tm + 1));
    B2P_CUDA(ctx, w->t_rowptr.reserve(tn + 1));
    for (auto* bf : {&w->colidx, &w->t_colidx}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->vals, &w->t_vals, &w->sv64, &w->stv64}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->sv32, &w->stv32}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->dr, &w->pu}) B2P_CUDA(ctx, bf->reserve(tm));
    for (auto* bf : {&w->dc, &w->pv}) B2P_CUDA(ctx, bf->reserve(tn));
    B2P_CUDA(ctx, w->r_ext.reserve(tm));
    B2P_CUDA(ctx, w->c_ext.reserve(tn));
    for (auto* bf : {&w->mat_m, &w->mat_n}) B2P_CUDA(ctx, bf->reserve(nmat));
    for (auto* bf : {&w->mat_row_off, &w->mat_col_off, &w->mat_rs_off, &w->mat_cs_off}) B2P_CUDA(ctx, bf->reserve(nmat));
    B2P_CUDA(ctx, w->r_sptr.reserve(r_sptr.size()));
    B2P_CUDA(ctx, w->c_sptr.reserve(c_sptr.size()));
    B2P_CUDA(ctx, w->r_eidx.reserve(r_pad));
    B2P_CUDA(ctx, w->c_eidx.reserve(c_pad));
    B2P_CUDA(ctx, w->r_ev64.reserve(r_pad));
    B2P_CUDA(ctx, w->c_ev64.reserve(c_pad));
    B2P_CUDA(ctx, w->r_ev32.reserve(r_pad));
    B2P_CUDA(ctx, w->c_ev32.reserve(c_pad));
    B2P_CUDA(ctx, w->mat_eta.reserve(nmat));
    B2P_CUDA(ctx, w->inst_mat.reserve(count));
    for (auto* bf : {&w->x_off, &w->y_off}) B2P_CUDA(ctx, bf->reserve(count));
    for (auto* bf : {&w->c, &w->lb, &w->ub, &w->x, &w->xt}) B2P_CUDA(ctx, bf->reserve(IN));
    for (auto* bf : {&w->b, &w->y, &w->yt}) B2P_CUDA(ctx, bf->reserve(IM));
    B2P_CUDA(ctx, w->colp.reserve(4 * IN));
    B2P_CUDA(ctx, w->rowp.reserve(4 * IM));
    B2P_CUDA(ctx, w->is_eq.reserve(IM));
    for (auto* bf : {&w->bnorm, &w->cnorm}) B2P_CUDA(ctx, bf->reserve(count));
    B2P_CUDA(ctx, w->ictrl.reserve(count));
    for (auto* bf : {&w->active, &w->active2}) B2P_CUDA(ctx, bf->reserve(count));
    B2P_CUDA(ctx, w->counters.reserve(2));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->rowptr.p, grp.data(), sizeof(int32_t) * (tm + 1), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->colidx.p, gci.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->vals.p, gval.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->r_ext.p, r_ext.data(), sizeof(int32_t) * tm, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->c_ext.p, c_ext.data(), sizeof(int32_t) * tn, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->r_sptr.p, r_sptr.data(), sizeof(int64_t) * r_sptr.size(), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->c_sptr.p, c_sptr.data(), sizeof(int64_t) * c_sptr.size(), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_rs_off.p, rs_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_cs_off.p, cs_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_m.p, mat_m, sizeof(int32_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_n.p, mat_n, sizeof(int32_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_row_off.p, row_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_col_off.p, col_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->inst_mat.p, inst_mat, sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->x_off.p, xoff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->y_off.p, yoff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
    {
        // per-instance vectors arrive in external order: stage, then permute on the device
        DBuf<double> sb, scv, sl, su;
        DBuf<uint8_t> seq;
        for (auto* bf : {&scv, &sl, &su}) B2P_CUDA(ctx, bf->reserve(IN));
        B2P_CUDA(ctx, sb.reserve(IM));
        B2P_CUDA(ctx, seq.reserve(IM));
        B2P_CUDA(ctx, cudaMemcpyAsync(scv.p, c, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(sl.p, lb, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(su.p, ub, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(sb.p, b, sizeof(double) * IM, cudaMemcpyHostToDevice, s));
        B2P_CUDA(ctx, cudaMemcpyAsync(seq.p, is_eq, IM, cudaMemcpyHostToDevice, s));
        k_permute_inst<<<std::min(count, ctx->sm_count * 8), 256, 0, s>>>(
            count, w->inst_mat.p, w->mat_m.p, w->mat_n.p, w->mat_row_off.p, w->mat_col_off.p, w->x_off.p, w->y_off.p,
            w->r_ext.p, w->c_ext.p, sb.p, scv.p, sl.p, su.p, seq.p, w->b.p, w->c.p, w->lb.p, w->ub.p, w->is_eq.p);
        B2P_LAUNCH(ctx);
        ctx->launches += 1;
        B2P_CUDA(ctx, cudaStreamSynchronize(s));  // staging buffers are released at scope end
    }
    int st = build_transpose(ctx, (int)tm, (int)tn, nnz, w->rowptr.p, w->colidx.p, w->vals.p, w->t_rowptr.p,
                             w->t_colidx.p, w->t_vals.p);
    if (st) return st;
    // scaling + scaled values + step sizes (per matrix, FP64), then the SELL-32 copies
    DBuf<double> tr, tc;
    B2P_CUDA(ctx, tr.reserve(tm));
    B2P_CUDA(ctx, tc.reserve(tn));
    int ruiz = 10;
    int gmat = std::min(nmat, ctx->sm_count * 8);
    k_batch_scaling<<<gmat, 256, 0, s>>>(nmat, w->mat_m.p, w->mat_n.p, w->mat_row_off.p, w->mat_col_off.p, w->rowptr.p,
                                          w->colidx.p, w->vals.p, w->t_rowptr.p, w->t_colidx.p, w->t_vals.p, ruiz,
                                          w->dr.p, w->dc.p, tr.p, tc.p);
    k_batch_scale_vals<<<grid_for(std::max(tm, tn), 256, ctx->sm_count), 256, 0, s>>>(
        tm, tn, w->rowptr.p, w->colidx.p, w->vals.p, w->t_rowptr.p, w->t_colidx.p, w->t_vals.p, w->dr.p, w->dc.p,
        w->sv64.p, w->sv32.p, w->stv64.p, w->stv32.p);
    k_batch_power<<<gmat, 256, 0, s>>>(nmat, w->mat_m.p, w->mat_n.p, w->mat_row_off.p, w->mat_col_off.p, w->rowptr.p,
                                        w->colidx.p, w->sv64.p, w->t_rowptr.p, w->t_colidx.p, w->stv64.p, w->pv.p,
                                        w->pu.p, 0.998, w->mat_eta.p);
    k_fill_ell<<<gmat, 256, 0, s>>>(1, nmat, w->mat_m.p, w->mat_row_off.p, w->mat_col_off.p, w->mat_rs_off.p, w->r_sptr.p,
                                     w->rowptr.p, w->colidx.p, w->sv64.p, w->sv32.p, w->r_eidx.p, w->r_ev64.p,
                                     w->r_ev32.p);
    k_fill_ell<<<gmat, 256, 0, s>>>(1, nmat, w->mat_n.p, w->mat_col_off.p, w->mat_row_off.p, w->mat_cs_off.p, w->c_sptr.p,
                                     w->t_rowptr.p, w->t_colidx.p, w->stv64.p, w->stv32.p, w->c_eidx.p, w->c_ev64.p,
                                     w->c_ev32.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 5;
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    return B2P_OK;
}

int b2p_batch_solve(void* p, const b2p_params* params, const double* x0, const double* y0, const double* omega0,
                    int32_t* status_out, int64_t* iters_out, double* kkt_out, double* omega_out, double* x_out,
                    double* y_out, b2p_result* summary) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    BatchWork* w = ctx->bw;
    if (!w) {
        ctx->err = "b2p_batch_solve: no batch uploaded";
        return B2P_NO_LP;
    }
    b2p_params def;
    b2p_params_default(&def);
    def.engine = B2P_ENGINE_HALPERN;
    const b2p_params* pp = params ? params : &def;
    if (pp->check_every < 2 || pp->max_iterations < 0) {
        ctx->err = "b2p_batch_solve: check_every must be >= 2";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    if (summary) std::memset(summary, 0, sizeof(*summary));
    int64_t l0 = ctx->launches;
    double t0 = now_ms();
    cudaStream_t s = ctx->stream;
    // warm starts / weights to the device
    DBuf<double> dx0, dy0, dom;
    if (x0) {
        B2P_CUDA(ctx, dx0.reserve(w->inst_n));
        B2P_CUDA(ctx, cudaMemcpyAsync(dx0.p, x0, sizeof(double) * w->inst_n, cudaMemcpyHostToDevice, s));
    }
    if (y0) {
        B2P_CUDA(ctx, dy0.reserve(w->inst_m));
        B2P_CUDA(ctx, cudaMemcpyAsync(dy0.p, y0, sizeof(double) * w->inst_m, cudaMemcpyHostToDevice, s));
    }
    if (omega0) {
        B2P_CUDA(ctx, dom.reserve(w->count));
        B2P_CUDA(ctx, cudaMemcpyAsync(dom.p, omega0, sizeof(double) * w->count, cudaMemcpyHostToDevice, s));
    }
    bool timed_out = false;
    float kms = 0.0f;
    TuneCfg cfg = {0, 0};
    int st = pp->precision == B2P_FP64
                 ? batch_run<double>(ctx, w, pp, x0 ? dx0.p : nullptr, y0 ? dy0.p : nullptr, omega0 ? dom.p : nullptr,
                                     nullptr, &timed_out, &kms, &cfg)
                 : batch_run<float>(ctx, w, pp, x0 ? dx0.p : nullptr, y0 ? dy0.p : nullptr, omega0 ? dom.p : nullptr,
                                    nullptr, &timed_out, &kms, &cfg);
    if (st) return st;
    int64_t tot_it, maxit, opt;
    double worst;
    st = collect_outputs(ctx, w, timed_out, status_out, iters_out, kkt_out, omega_out, x_out, y_out, &tot_it, &maxit,
                         &opt, &worst);
    if (st) return st;
    fill_summary(summary, w->count, timed_out, tot_it, maxit, opt, worst, kms, cfg);
    if (summary) {
        summary->solve_time_ms = now_ms() - t0;
        summary->kernel_launches = ctx->launches - l0;
    }
    return B2P_OK;
}

int b2p_batch_trace(void* p, int capacity, int* count, double* t_ms, int32_t* active) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    BatchWork* w = ctx->bw;
    if (!w || !w->solved) {
        ctx->err = "b2p_batch_trace: no batched solve to report";
        return B2P_NO_LP;
    }
    const int n = (int)w->trace_ms.size();
    if (count) *count = n;
    const int k = std::min(n, std::max(capacity, 0));
    for (int i = 0; i < k; ++i) {
        if (t_ms) t_ms[i] = w->trace_ms[i];
        if (active) active[i] = w->trace_active[i];
    }
    return B2P_OK;
}

int b2p_batch_objectives(void* p, double* pobj_out, double* dobj_out, double* obj_err_out) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    BatchWork* w = ctx->bw;
    if (!w || !w->solved || (int)w->hc.size() != w->count) {
        ctx->err = "b2p_batch_objectives: no batched solve to report";
        return B2P_NO_LP;
    }
    for (int i = 0; i < w->count; ++i) {
        if (pobj_out) pobj_out[i] = w->hc[i].pobj;
        if (dobj_out) dobj_out[i] = w->hc[i].dobj;
        if (obj_err_out) obj_err_out[i] = w->hc[i].obj_err;
    }
    return B2P_OK;
}

int b2p_batch_solve_learned(void* p, const b2p_params* params, const float* features, int fallback,
                            int32_t* status_out, int64_t* iters_out, double* kkt_out, uint8_t* warm_used_out,
                            double* x_out, double* y_out, b2p_result* summary) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    BatchWork* w = ctx->bw;
    if (!w) {
        ctx->err = "b2p_batch_solve_learned: no batch uploaded";
        return B2P_NO_LP;
    }
    if (!features) {
        ctx->err = "b2p_batch_solve_learned: null parameter vectors";
        return B2P_INVALID_ARGUMENT;
    }
    int n = 0, m = 0;
    if (!uniform_shape(w, &n, &m)) {
        ctx->err = "b2p_batch_solve_learned: the instances of the batch differ in shape";
        return B2P_INVALID_ARGUMENT;
    }
    b2p_params def;
    b2p_params_default(&def);
    def.engine = B2P_ENGINE_HALPERN;
    def.precision = B2P_FP32;
    const b2p_params* pp = params ? params : &def;
    if (pp->check_every < 2 || pp->max_iterations < 0) {
        ctx->err = "b2p_batch_solve_learned: check_every must be >= 2";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    if (summary) std::memset(summary, 0, sizeof(*summary));
    int64_t l0 = ctx->launches;
    double t0 = now_ms();
    // warm start from the MLP, on the device
    DBuf<double> dx0, dy0, dom;
    B2P_CUDA(ctx, dx0.reserve(w->inst_n));
    B2P_CUDA(ctx, dy0.reserve(w->inst_m));
    B2P_CUDA(ctx, dom.reserve(w->count));
    int st = mlp_predict_warm(ctx, features, w->count, n, m, dx0.p, dy0.p, dom.p);
    if (st) return st;
    const bool f64 = pp->precision == B2P_FP64;
    bool timed_out = false;
    float kms = 0.0f, kms2 = 0.0f;
    TuneCfg cfg = {0, 0};
    st = f64 ? batch_run<double>(ctx, w, pp, dx0.p, dy0.p, dom.p, nullptr, &timed_out, &kms, &cfg)
             : batch_run<float>(ctx, w, pp, dx0.p, dy0.p, dom.p, nullptr, &timed_out, &kms, &cfg);
    if (st) return st;
    // cold-start fallback for every instance the warm-started run did not solve and
    // that has iterations left: the cold run continues the instance's iteration count,
    // so warm + cold together stay within max_iterations (an instance that spent its
    // whole budget warm is reported MAX_ITERATIONS, as a cold run would be)
    std::vector<long long> warm_iters(w->count);
    std::vector<int32_t> failed;
    for (int i = 0; i < w->count; ++i) {
        warm_iters[i] = w->hc[i].total;
        // an answer, or a certificate of infeasibility / unboundedness (which holds
        // whatever the starting point), ends the instance
        const int sti = w->hc[i].status;
        const bool ok = w->hc[i].done && (sti == B2P_STATUS_OPTIMAL || sti == B2P_STATUS_INFEASIBLE_DETECTED ||
                                          sti == B2P_STATUS_UNBOUNDED_DETECTED);
        if (!ok && warm_iters[i] < pp->max_iterations) failed.push_back(i);
    }
    if (fallback && !failed.empty() && !timed_out) {
        st = f64 ? batch_run<double>(ctx, w, pp, nullptr, nullptr, nullptr, &failed, &timed_out, &kms2, &cfg,
                                     &warm_iters)
                 : batch_run<float>(ctx, w, pp, nullptr, nullptr, nullptr, &failed, &timed_out, &kms2, &cfg,
                                    &warm_iters);
        if (st) return st;
    }
    int64_t tot_it, maxit, opt;
    double worst;
    // iterations per instance: the warm run, plus the cold run when it fell back
    st = collect_outputs(ctx, w, timed_out, status_out, iters_out, kkt_out, nullptr, x_out, y_out, &tot_it, &maxit,
                         &opt, &worst);
    if (st) return st;
    std::vector<uint8_t> is_failed(w->count, 0);
    if (fallback)
        for (int32_t i : failed) is_failed[i] = 1;
    if (warm_used_out)
        for (int i = 0; i < w->count; ++i) warm_used_out[i] = is_failed[i] ? 0 : 1;
    fill_summary(summary, w->count, timed_out, tot_it, maxit, opt, worst, kms + kms2, cfg);
    if (summary) {
        summary->solve_time_ms = now_ms() - t0;
        summary->kernel_launches = ctx->launches - l0;
        summary->refinement_rounds_done = fallback ? (int)failed.size() : 0;  // instances that fell back
    }
    return B2P_OK;
}

int b2p_mlp_dataset_from_batch(void* p, const float* features, int count) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    BatchWork* w = ctx->bw;
    if (!w || !w->solved) {
        ctx->err = "b2p_mlp_dataset_from_batch: no solved batch";
        return B2P_NO_LP;
    }
    if (!features || count != w->count) {
        ctx->err = "b2p_mlp_dataset_from_batch: one parameter vector per instance of the batch is required";
        return B2P_INVALID_ARGUMENT;
    }
    int n = 0, m = 0;
    if (!uniform_shape(w, &n, &m)) {
        ctx->err = "b2p_mlp_dataset_from_batch: the instances of the batch differ in shape";
        return B2P_INVALID_ARGUMENT;
    }
    cudaSetDevice(ctx->device);
    return mlp_set_dataset(ctx, features, count, n, m, w->ox.p, w->oy.p, w->oom.p);
}

}  // extern "C"
