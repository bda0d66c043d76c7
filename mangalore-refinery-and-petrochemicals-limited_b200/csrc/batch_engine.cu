// Batched engine: thousands of independent LPs in one persistent launch.
//
// Layout in HBM
//   * `nmat` constraint matrices concatenated into one block-diagonal CSR with
//     GLOBAL row/column indices (row_off[k], col_off[k] per matrix) plus its
//     stable transpose; FP64 originals, FP64 and FP32 scaled copies.
//   * `count` instances, each naming a matrix; per-instance vectors (b, c, l, u
//     in FP64 for the KKT; scaled FP32/FP64 copies; iterates x, xa, xt, y, ya,
//     yt) concatenated at x_off[i] / y_off[i].
// Execution
//   * one CTA owns one instance at a time (persistent grid, work queue sorted by
//     nnz descending = longest-first).  The gathered operands of both SpMVs --
//     y (FP64, also the dual iterate) for A^T y and xh for A xh -- live in shared
//     memory; x and the anchors stay in global memory, touched only by their
//     owning lane.  A PDHG iteration is: primal phase (columns, LC lanes each) |
//     barrier | dual phase (rows, LR lanes each) | barrier, with matrix entries
//     streamed from L2/HBM and every gather served from shared memory.
//   * precision as in the single-LP engine: MT (float = mixed, double = FP64) is
//     the storage type of the scaled matrix values and of xh; iterates, sums,
//     scaling and the KKT are FP64.
//   * per instance: own step size (from its matrix), primal weight, Halpern
//     counter, restart state, FP64 KKT every K iterations (block reductions in a
//     fixed order: deterministic), own termination.
//   * a launch runs every active instance for up to `chunk` iterations; a
//     compaction kernel drops finished instances; [reset, chunk, compact] is
//     captured as a CUDA graph and replayed until no instance is active.
//   * lanes per column / row, block size and chunk length come from an
//     autotuner that times candidates on a sample of the batch (cached on disk).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
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
    long long k, total, restarts;
    int status, done, first;
    int pad;
};

struct BatchWork {
    int nmat = 0, count = 0;
    int64_t tot_m = 0, tot_n = 0, nnz = 0, inst_m = 0, inst_n = 0;
    // matrices
    DBuf<int32_t> rowptr, colidx, t_rowptr, t_colidx;
    DBuf<double> vals, t_vals, sv64, stv64, dr, dc, pv, pu;
    DBuf<float> sv32, stv32;
    DBuf<int32_t> mat_m, mat_n;
    DBuf<int64_t> mat_row_off, mat_col_off;
    DBuf<double> mat_eta;
    std::vector<int32_t> h_mat_m, h_mat_n;
    std::vector<int64_t> h_mat_nnz;
    // instances
    DBuf<int32_t> inst_mat;
    DBuf<int64_t> x_off, y_off;
    DBuf<double> b, c, lb, ub, bnorm, cnorm;
    DBuf<uint8_t> is_eq;
    DBuf<double> bs, cs, ls, us, x, xa, xt, y, ya, yt;  // scaled vectors and FP64 iterates
    bool recenter = false;
    DBuf<double> xbar, atybar, ybar, axbar, ylb_s;      // re-centring state (per instance)
    DBuf<InstCtrl> ictrl;
    DBuf<int32_t> active, active2, counters;  // counters[0]=head, [1]=active count
    std::vector<int32_t> h_inst_mat, order;
    int max_m = 0, max_n = 0;
};

void batch_free(Ctx* ctx) {
    delete ctx->bw;
    ctx->bw = nullptr;
}

namespace {

struct BArgs {
    // matrices
    const int32_t *rowptr, *colidx, *t_rowptr, *t_colidx;
    const double *sv64, *stv64, *dr, *dc, *mat_eta;
    const void *sv, *stv;  // T-typed scaled values
    const int32_t *mat_m, *mat_n;
    const int64_t *mat_row_off, *mat_col_off;
    // instances
    const int32_t* inst_mat;
    const int64_t *x_off, *y_off;
    const double *b, *c, *lb, *ub, *bnorm, *cnorm;
    const uint8_t* is_eq;
    double *bs, *cs, *ls, *us;  // scaled problem vectors (rewritten by re-centring)
    double *x, *xa, *xt, *y, *ya, *yt;
    InstCtrl* ictrl;
    const int32_t* active;
    int32_t* counters;
    // parameters
    double eps, beta_s, beta_n, beta_a, rho;
    // FP64 re-centring at restarts (as in the single-LP engine): per-instance centre in
    // the original space, A xbar, A^T ybar, shifted dual bound; original FP64 values
    int recenter;
    const double *vals, *t_vals;
    double *xbar, *ybar, *axbar, *atybar, *ylb_s;
    long long max_iter;
    int K;
};

template <typename T>
__device__ __forceinline__ T clampT(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Block-wide FP64 sum of up to 6 values, fixed reduction order (deterministic).
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

template <typename MT, int LC, int LR>
__global__ void __launch_bounds__(512) k_batch_chunk(BArgs a, int chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32 * 6];
    __shared__ InstCtrl sc;
    __shared__ int s_q;
    __shared__ int s_flags[4];  // 0: done, 1: restart
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const MT* sv = (const MT*)a.sv;
    const MT* stv = (const MT*)a.stv;
    double *bs = a.bs, *cs = a.cs, *ls = a.ls, *us = a.us;
    double *xg = a.x, *xag = a.xa, *xtg = a.xt, *yg = a.y, *yag = a.ya, *ytg = a.yt;
    const int active_count = a.counters[1];
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
        const double eta = a.mat_eta[mat];
        double* ys = (double*)smem_raw;
        MT* xhs = (MT*)(ys + ((m + 1) & ~1));
        if (tid == 0) sc = a.ictrl[inst];
        for (int i = tid; i < m; i += nt) ys[i] = yg[yo + i];
        __syncthreads();
        const double rho = a.rho;
        for (int it = 0; it < chunk; ++it) {
            const long long kk = sc.k;
            const bool first = sc.first != 0;
            const bool check = ((sc.total + 1) % a.K) == 0;
            const double om = sc.omega;
            const double tau = eta / om, sigma = eta * om;
            const double wk = (kk + 1.0) / (kk + 2.0), wa = 1.0 / (kk + 2.0);
            double acc[6] = {0, 0, 0, 0, 0, 0};  // rx2 (first or check), dxa2, ry2, dya2
            // ---- primal phase: columns (gathers y from shared memory)
            {
                const int sub = lane & (LC - 1), per_warp = 32 / LC;
                for (int base = warp * per_warp; base < n; base += nwarps * per_warp) {
                    const int j = base + lane / LC;
                    const bool valid = j < n;
                    double s = 0.0;
                    if (valid) {
                        const int64_t gj = co + j;
                        const int e1 = a.t_rowptr[gj + 1];
                        for (int e = a.t_rowptr[gj] + sub; e < e1; e += LC) s += (double)stv[e] * ys[a.t_colidx[e] - ro];
                    }
#pragma unroll
                    for (int o = LC / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (valid && sub == 0) {
                        const double xj = xg[xo + j];
                        const double xt = clampT(xj - tau * (cs[xo + j] + s), ls[xo + j], us[xo + j]);
                        xhs[j] = (MT)(2.0 * xt - xj);
                        const double xa = xag[xo + j];
                        xg[xo + j] = wk * ((1.0 + rho) * xt - rho * xj) + wa * xa;
                        if (first || check) {
                            double d = xj - xt;
                            acc[0] += d * d;
                        }
                        if (check) {
                            xtg[xo + j] = xt;
                            double e = xt - xa;
                            acc[1] += e * e;
                        }
                    }
                }
            }
            __syncthreads();
            // ---- dual phase: rows (gathers xh from shared memory)
            {
                const int sub = lane & (LR - 1), per_warp = 32 / LR;
                for (int base = warp * per_warp; base < m; base += nwarps * per_warp) {
                    const int i = base + lane / LR;
                    const bool valid = i < m;
                    double s = 0.0;
                    if (valid) {
                        const int64_t gi = ro + i;
                        const int e1 = a.rowptr[gi + 1];
                        for (int e = a.rowptr[gi] + sub; e < e1; e += LR) s += (double)sv[e] * (double)xhs[a.colidx[e] - co];
                    }
#pragma unroll
                    for (int o = LR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (valid && sub == 0) {
                        const double yi = ys[i];
                        double yt = yi + sigma * (s - bs[yo + i]);
                        if (!a.is_eq[yo + i]) {
                            const double lbv = a.recenter ? a.ylb_s[yo + i] : 0.0;
                            if (yt < lbv) yt = lbv;
                        }
                        const double ya = yag[yo + i];
                        ys[i] = wk * ((1.0 + rho) * yt - rho * yi) + wa * ya;
                        if (first || check) {
                            double d = yi - yt;
                            acc[2] += d * d;
                        }
                        if (check) {
                            ytg[yo + i] = yt;
                            double e = yt - ya;
                            acc[3] += e * e;
                        }
                    }
                }
            }
            if (first || check) block_sums<6>(acc, red);
            __syncthreads();
            if (tid == 0) {
                if (first) {
                    sc.r0 = sqrt(om * acc[0] + acc[2] / om);
                    sc.rprev = sc.r0;
                    sc.first = 0;
                }
                sc.k += 1;
                sc.total += 1;
                s_flags[0] = 0;
                s_flags[1] = 0;
            }
            if (!check) {
                __syncthreads();
                continue;
            }
            // restart residuals (thread 0 holds the block sums)
            double r_now = 0, dxa = 0, dya = 0;
            if (tid == 0) {
                r_now = sqrt(om * acc[0] + acc[2] / om);
                dxa = sqrt(acc[1]);
                dya = sqrt(acc[3]);
            }
            __syncthreads();  // xt / yt of this iteration are in global memory
            // ---- FP64 KKT of T(z) on the original instance
            double kk2[6] = {0, 0, 0, 0, 0, 0};  // pres2, by, dres2, pc, lam
            {
                const int sub = lane & (LR - 1), per_warp = 32 / LR;
                for (int base = warp * per_warp; base < m; base += nwarps * per_warp) {
                    const int i = base + lane / LR;
                    const bool valid = i < m;
                    double s = 0.0;
                    if (valid) {
                        const int64_t gi = ro + i;
                        for (int e = a.rowptr[gi] + sub; e < a.rowptr[gi + 1]; e += LR)
                            s += a.sv64[e] * xtg[xo + a.colidx[e] - co];
                    }
#pragma unroll
                    for (int o = LR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (valid && sub == 0) {
                        const double dri = a.dr[ro + i];
                        const double ax = (a.recenter ? a.axbar[yo + i] : 0.0) + s / dri;
                        double rp = ax - a.b[yo + i];
                        if (!a.is_eq[yo + i]) rp = fmax(rp, 0.0);
                        kk2[0] += rp * rp;
                        kk2[1] += a.b[yo + i] * ((a.recenter ? a.ybar[yo + i] : 0.0) + dri * ytg[yo + i]);
                    }
                }
            }
            {
                const int sub = lane & (LC - 1), per_warp = 32 / LC;
                for (int base = warp * per_warp; base < n; base += nwarps * per_warp) {
                    const int j = base + lane / LC;
                    const bool valid = j < n;
                    double s = 0.0;
                    if (valid) {
                        const int64_t gj = co + j;
                        for (int e = a.t_rowptr[gj] + sub; e < a.t_rowptr[gj + 1]; e += LC)
                            s += a.stv64[e] * ytg[yo + a.t_colidx[e] - ro];
                    }
#pragma unroll
                    for (int o = LC / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (valid && sub == 0) {
                        const double dcj = a.dc[co + j];
                        const double cj = a.c[xo + j], lj = a.lb[xo + j], uj = a.ub[xo + j];
                        const double g = cj + (a.recenter ? a.atybar[xo + j] : 0.0) + s / dcj;
                        const bool fl = isfinite(lj), fu = isfinite(uj);
                        const double lam = (fl && fu) ? g : (fl ? fmax(g, 0.0) : (fu ? fmin(g, 0.0) : 0.0));
                        const double rd = g - lam;
                        kk2[2] += rd * rd;
                        kk2[3] += cj * ((a.recenter ? a.xbar[xo + j] : 0.0) + dcj * xtg[xo + j]);
                        if (lam > 0.0) kk2[4] += lam * lj;
                        else if (lam < 0.0) kk2[4] += lam * uj;
                    }
                }
            }
            block_sums<6>(kk2, red);
            if (tid == 0) {
                const double pres = sqrt(kk2[0]), dres = sqrt(kk2[2]);
                const double pobj = kk2[3], dobj = -kk2[1] + kk2[4];
                sc.rel_p = pres / (1.0 + a.bnorm[inst]);
                sc.rel_d = dres / (1.0 + a.cnorm[inst]);
                sc.rel_g = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
                sc.pobj = pobj;
                sc.dobj = dobj;
                const bool finite = isfinite(pres) && isfinite(dres) && isfinite(pobj) && isfinite(dobj) && isfinite(r_now);
                if (!finite) {
                    sc.done = 1;
                    sc.status = B2P_STATUS_NUMERICAL_FAILURE;
                } else if (sc.rel_p <= a.eps && sc.rel_d <= a.eps && sc.rel_g <= a.eps) {
                    sc.done = 1;
                    sc.status = B2P_STATUS_OPTIMAL;
                } else if (sc.total >= a.max_iter) {
                    sc.done = 1;
                    sc.status = B2P_STATUS_MAX_ITERATIONS;
                }
                if (!sc.done) {
                    const bool rs = (r_now <= a.beta_s * sc.r0) || (r_now <= a.beta_n * sc.r0 && r_now > sc.rprev) ||
                                    ((double)sc.k >= a.beta_a * (double)sc.total);
                    sc.rprev = r_now;
                    if (rs) {
                        if (dxa > 1e-10 && dya > 1e-10) {
                            const double nw = exp(0.5 * log(dya / dxa) + 0.5 * log(om));
                            if (isfinite(nw) && nw > 0.0) sc.omega = nw;
                        }
                        sc.k = 0;
                        sc.first = 1;
                        sc.restarts += 1;
                        s_flags[1] = 1;
                    }
                }
                s_flags[0] = sc.done;
            }
            __syncthreads();
            if (s_flags[1] && !a.recenter) {  // restart: z <- anchor <- T(z)
                for (int j = tid; j < n; j += nt) {
                    const double v = xtg[xo + j];
                    xg[xo + j] = v;
                    xag[xo + j] = v;
                }
                for (int i = tid; i < m; i += nt) {
                    const double v = ytg[yo + i];
                    ys[i] = v;
                    yag[yo + i] = v;
                }
            } else if (s_flags[1]) {
                // restart with re-centring: the LP is rewritten around T(z) (an exact change of
                // variables) with b - A xbar and c + A^T ybar from the FP64 original matrix
                for (int j = tid; j < n; j += nt) {
                    a.xbar[xo + j] += a.dc[co + j] * xtg[xo + j];
                    xg[xo + j] = 0.0;
                    xag[xo + j] = 0.0;
                    xtg[xo + j] = 0.0;
                }
                for (int i = tid; i < m; i += nt) {
                    a.ybar[yo + i] += a.dr[ro + i] * ytg[yo + i];
                    ys[i] = 0.0;
                    yag[yo + i] = 0.0;
                    ytg[yo + i] = 0.0;
                }
                __syncthreads();
                for (int i = tid; i < m; i += nt) {
                    const int64_t gi = ro + i;
                    double s = 0.0;
                    for (int e = a.rowptr[gi]; e < a.rowptr[gi + 1]; ++e) s += a.vals[e] * a.xbar[xo + a.colidx[e] - co];
                    const double dri = a.dr[gi];
                    a.axbar[yo + i] = s;
                    bs[yo + i] = dri * (a.b[yo + i] - s);
                    a.ylb_s[yo + i] = -a.ybar[yo + i] / dri;
                }
                for (int j = tid; j < n; j += nt) {
                    const int64_t gj = co + j;
                    double s = 0.0;
                    for (int e = a.t_rowptr[gj]; e < a.t_rowptr[gj + 1]; ++e)
                        s += a.t_vals[e] * a.ybar[yo + a.t_colidx[e] - ro];
                    const double dcj = a.dc[gj];
                    a.atybar[xo + j] = s;
                    cs[xo + j] = dcj * (a.c[xo + j] + s);
                    ls[xo + j] = (a.lb[xo + j] - a.xbar[xo + j]) / dcj;
                    us[xo + j] = (a.ub[xo + j] - a.xbar[xo + j]) / dcj;
                }
            }
            __syncthreads();
            if (s_flags[0]) break;
        }
        // store the dual iterate and the control block
        for (int i = tid; i < m; i += nt) yg[yo + i] = ys[i];
        if (tid == 0) a.ictrl[inst] = sc;
        __syncthreads();
    }
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

__global__ void k_copy_i32(int n, const int32_t* __restrict__ a, int32_t* __restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
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
        double est = 0.0;
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
                est = nn;
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

// per-instance scaled vectors, norms, initial point and control block (CTA per instance)
template <typename T>
__global__ void k_batch_init(int count, const int32_t* __restrict__ inst_mat, const int32_t* __restrict__ mat_m,
                             const int32_t* __restrict__ mat_n, const int64_t* __restrict__ row_off,
                             const int64_t* __restrict__ col_off, const int64_t* __restrict__ x_off,
                             const int64_t* __restrict__ y_off, const double* __restrict__ dr,
                             const double* __restrict__ dc, const double* __restrict__ b, const double* __restrict__ c,
                             const double* __restrict__ lb, const double* __restrict__ ub,
                             const uint8_t* __restrict__ is_eq, const double* __restrict__ x0,
                             const double* __restrict__ y0, const double* __restrict__ omega0, T* bs, T* cs, T* ls,
                             T* us, T* x, T* xa, T* xt, T* y, T* ya, T* yt, double* bnorm, double* cnorm,
                             InstCtrl* ictrl) {
    __shared__ double red[32 * 4];
    for (int inst = blockIdx.x; inst < count; inst += gridDim.x) {
        const int k = inst_mat[inst];
        const int m = mat_m[k], n = mat_n[k];
        const int64_t ro = row_off[k], co = col_off[k], xo = x_off[inst], yo = y_off[inst];
        double acc[4] = {0, 0, 0, 0};  // ||b||^2, ||c||^2, ||b_s||^2, ||c_s||^2
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double d = dc[co + j];
            const double cj = c[xo + j], csj = cj * d;
            const T l = (T)(lb[xo + j] / d), u = (T)(ub[xo + j] / d);
            cs[xo + j] = (T)csj;
            ls[xo + j] = l;
            us[xo + j] = u;
            T v = x0 ? (T)(x0[xo + j] / d) : (T)0;
            v = clampT(v, l, u);
            x[xo + j] = v;
            xa[xo + j] = v;
            xt[xo + j] = v;
            acc[1] += cj * cj;
            acc[3] += csj * csj;
        }
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const double d = dr[ro + i];
            const double bi = b[yo + i], bsi = bi * d;
            bs[yo + i] = (T)bsi;
            T v = y0 ? (T)(y0[yo + i] / d) : (T)0;
            if (!is_eq[yo + i] && v < (T)0) v = (T)0;
            y[yo + i] = v;
            ya[yo + i] = v;
            yt[yo + i] = v;
            acc[0] += bi * bi;
            acc[2] += bsi * bsi;
        }
        block_sums<4>(acc, red);
        if (threadIdx.x == 0) {
            bnorm[inst] = sqrt(acc[0]);
            cnorm[inst] = sqrt(acc[1]);
            const double bn = sqrt(acc[2]), cn = sqrt(acc[3]);
            InstCtrl s;
            memset(&s, 0, sizeof(s));
            s.omega = (omega0 && omega0[inst] > 0.0) ? omega0[inst] : ((bn > 1e-10 && cn > 1e-10) ? cn / bn : 1.0);
            s.first = 1;
            s.status = B2P_STATUS_MAX_ITERATIONS;
            ictrl[inst] = s;
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void k_batch_unscale(int count, const int32_t* __restrict__ inst_mat, const int32_t* __restrict__ mat_m,
                                const int32_t* __restrict__ mat_n, const int64_t* __restrict__ row_off,
                                const int64_t* __restrict__ col_off, const int64_t* __restrict__ x_off,
                                const int64_t* __restrict__ y_off, const double* __restrict__ dr,
                                const double* __restrict__ dc, const T* __restrict__ xt, const T* __restrict__ yt,
                                const double* __restrict__ xbar, const double* __restrict__ ybar,
                                double* __restrict__ xo_, double* __restrict__ yo_) {
    for (int inst = blockIdx.x; inst < count; inst += gridDim.x) {
        const int k = inst_mat[inst];
        const int m = mat_m[k], n = mat_n[k];
        const int64_t ro = row_off[k], co = col_off[k], xo = x_off[inst], yo = y_off[inst];
        for (int j = threadIdx.x; j < n; j += blockDim.x)
            xo_[xo + j] = (xbar ? xbar[xo + j] : 0.0) + dc[co + j] * (double)xt[xo + j];
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            yo_[yo + i] = (ybar ? ybar[yo + i] : 0.0) + dr[ro + i] * (double)yt[yo + i];
    }
}

// ------------------------------------------------------------------ host side
struct TuneCfg {
    int lc, lr, threads, chunk;
};

template <typename T>
using ChunkFn = void (*)(BArgs, int);

template <typename T>
ChunkFn<T> chunk_kernel(int lc, int lr) {
#define SEL(C_, R_) if (lc == C_ && lr == R_) return k_batch_chunk<T, C_, R_>;
    SEL(4, 8) SEL(4, 16) SEL(4, 32) SEL(8, 8) SEL(8, 16) SEL(8, 32) SEL(2, 8) SEL(2, 16) SEL(2, 32)
#undef SEL
    return k_batch_chunk<T, 4, 16>;
}

std::string cache_path() {
    const char* p = std::getenv("B2P_AUTOTUNE_CACHE");
    if (p && *p) return p;
    const char* h = std::getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/b2p_autotune.txt";
}

std::string batch_key(BatchWork* w, int precision) {
    // signature: precision, size classes of the batch
    double mean_m = (double)w->inst_m / w->count, mean_n = (double)w->inst_n / w->count;
    double nnz_col = (double)w->nnz / std::max<int64_t>(w->tot_n, 1);
    std::ostringstream os;
    os << "p" << precision << "_c" << (int)std::log2(std::max(1, w->count)) << "_m" << (int)std::log2(mean_m + 1)
       << "_n" << (int)std::log2(mean_n + 1) << "_k" << (int)std::lround(nnz_col) << "_M" << w->max_m << "_N" << w->max_n
       << "_shared" << (w->nmat == 1 && w->count > 1);
    return os.str();
}

bool cache_lookup(const std::string& key, TuneCfg* out) {
    std::ifstream f(cache_path());
    std::string k;
    TuneCfg c;
    while (f >> k >> c.lc >> c.lr >> c.threads >> c.chunk)
        if (k == key) {
            *out = c;
            return true;
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
    f << key << " " << c.lc << " " << c.lr << " " << c.threads << " " << c.chunk << "\n";
}

BArgs make_args(BatchWork* w, const b2p_params* p, const void* sv, const void* stv, const int32_t* active) {
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
    a.sv = sv;
    a.stv = stv;
    a.mat_m = w->mat_m.p;
    a.mat_n = w->mat_n.p;
    a.mat_row_off = w->mat_row_off.p;
    a.mat_col_off = w->mat_col_off.p;
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
    a.bs = w->bs.p;
    a.cs = w->cs.p;
    a.ls = w->ls.p;
    a.us = w->us.p;
    a.x = w->x.p;
    a.xa = w->xa.p;
    a.xt = w->xt.p;
    a.y = w->y.p;
    a.ya = w->ya.p;
    a.yt = w->yt.p;
    a.ictrl = w->ictrl.p;
    a.active = active;
    a.counters = w->counters.p;
    a.eps = p->eps_rel_kkt;
    a.beta_s = p->restart_sufficient;
    a.beta_n = p->restart_necessary;
    a.beta_a = p->restart_artificial;
    a.rho = p->reflection;
    a.max_iter = p->max_iterations;
    a.K = p->check_every;
    a.recenter = w->recenter ? 1 : 0;
    a.vals = w->vals.p;
    a.t_vals = w->t_vals.p;
    a.xbar = w->xbar.p;
    a.ybar = w->ybar.p;
    a.axbar = w->axbar.p;
    a.atybar = w->atybar.p;
    a.ylb_s = w->ylb_s.p;
    return a;
}

// dynamic shared memory of one CTA: y (FP64) and xh (MT) of the largest instance
size_t smem_bytes(BatchWork* w, size_t mt_size) {
    return 8 * (size_t)((w->max_m + 1) & ~1) + mt_size * (size_t)w->max_n + 16;
}

int init_instances(Ctx* ctx, BatchWork* w, const double* x0_dev, const double* y0_dev, const double* om_dev) {
    int grid = std::min(w->count, ctx->sm_count * 8);
    k_batch_init<double><<<grid, 256, 0, ctx->stream>>>(
        w->count, w->inst_mat.p, w->mat_m.p, w->mat_n.p, w->mat_row_off.p, w->mat_col_off.p, w->x_off.p, w->y_off.p,
        w->dr.p, w->dc.p, w->b.p, w->c.p, w->lb.p, w->ub.p, w->is_eq.p, x0_dev, y0_dev, om_dev, w->bs.p, w->cs.p,
        w->ls.p, w->us.p, w->x.p, w->xa.p, w->xt.p, w->y.p, w->ya.p, w->yt.p, w->bnorm.p, w->cnorm.p, w->ictrl.p);
    B2P_LAUNCH(ctx);
    ctx->launches += 1;
    return B2P_OK;
}

template <typename MT>
const void* vals_of(BatchWork* w, bool transposed) {
    if (sizeof(MT) == 8) return transposed ? (const void*)w->stv64.p : (const void*)w->sv64.p;
    return transposed ? (const void*)w->stv32.p : (const void*)w->sv32.p;
}

// Times each candidate on a size-stratified sample of the batch (no termination,
// fixed iteration count); instance state is re-initialised afterwards by the caller.
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
    const int trial_iters = 128;
    std::vector<TuneCfg> cands;
    for (int lc : {2, 4, 8})
        for (int lr : {8, 16, 32})
            for (int th : {128, 256, 512}) cands.push_back({lc, lr, th, 2048});
    float best_ms = 1e30f;
    *best = {4, 16, 256, 2048};
    size_t sm = smem_bytes(w, sizeof(MT));
    for (const TuneCfg& c : cands) {
        int st = init_instances(ctx, w, nullptr, nullptr, nullptr);
        if (st) return st;
        int32_t cnt[2] = {0, sample};
        B2P_CUDA(ctx, cudaMemcpyAsync(w->counters.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s));
        BArgs a = make_args(w, &tp, vals_of<MT>(w, false), vals_of<MT>(w, true), dids.p);
        ChunkFn<MT> fn = chunk_kernel<MT>(c.lc, c.lr);
        B2P_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int per_sm = 0;
        B2P_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, c.threads, sm));
        if (per_sm < 1) continue;
        int grid = std::min(sample, ctx->sm_count * per_sm);
        cudaEventRecord(ctx->ev0, s);
        fn<<<grid, c.threads, sm, s>>>(a, trial_iters);
        cudaEventRecord(ctx->ev1, s);
        B2P_LAUNCH(ctx);
        B2P_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
        ctx->launches += 2;
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        if (ms < best_ms) {
            best_ms = ms;
            *best = c;
        }
    }
    cache_store(key, *best);
    return B2P_OK;
}

template <typename MT>
int batch_run(Ctx* ctx, BatchWork* w, const b2p_params* p, const double* x0, const double* y0, const double* omega0,
              int32_t* status_out, int64_t* iters_out, double* kkt_out, double* omega_out, double* x_out, double* y_out,
              b2p_result* sum) {
    cudaStream_t s = ctx->stream;
    double t_start = now_ms();
    const int64_t IN = w->inst_n, IM = w->inst_m;
    w->recenter = false;  // autotune trials run without re-centring (its buffers are set up below)
    // lanes per column / row, threads per CTA, chunk length: explicit, cached or tuned now
    TuneCfg cfg = {4, 16, 256, 2048};
    if (p->lanes_per_row > 0) {
        cfg.lc = std::min(8, std::max(2, p->lanes_per_row / 4));
        cfg.lr = p->lanes_per_row < 8 ? 8 : std::min(32, p->lanes_per_row);
    } else {
        int st = autotune<MT>(ctx, w, p, &cfg);
        if (st) return st;
    }
    // warm starts / weights
    DBuf<double> dx0, dy0, dom;
    if (x0) {
        B2P_CUDA(ctx, dx0.reserve(IN));
        B2P_CUDA(ctx, cudaMemcpyAsync(dx0.p, x0, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
    }
    if (y0) {
        B2P_CUDA(ctx, dy0.reserve(IM));
        B2P_CUDA(ctx, cudaMemcpyAsync(dy0.p, y0, sizeof(double) * IM, cudaMemcpyHostToDevice, s));
    }
    if (omega0) {
        B2P_CUDA(ctx, dom.reserve(w->count));
        B2P_CUDA(ctx, cudaMemcpyAsync(dom.p, omega0, sizeof(double) * w->count, cudaMemcpyHostToDevice, s));
    }
    int st = init_instances(ctx, w, x0 ? dx0.p : nullptr, y0 ? dy0.p : nullptr, omega0 ? dom.p : nullptr);
    if (st) return st;
    // re-centring: on by default for the mixed engine (refinement_rounds < 0), forced by > 0
    w->recenter = p->refinement_rounds > 0 || (p->refinement_rounds < 0 && sizeof(MT) == 4);
    if (w->recenter) {
        for (auto* b : {&w->xbar, &w->atybar}) {
            B2P_CUDA(ctx, b->reserve(IN));
            B2P_CUDA(ctx, cudaMemsetAsync(b->p, 0, sizeof(double) * IN, s));
        }
        for (auto* b : {&w->ybar, &w->axbar, &w->ylb_s}) {
            B2P_CUDA(ctx, b->reserve(IM));
            B2P_CUDA(ctx, cudaMemsetAsync(b->p, 0, sizeof(double) * IM, s));
        }
    }
    // active list = all instances, longest first
    B2P_CUDA(ctx, cudaMemcpyAsync(w->active.p, w->order.data(), sizeof(int32_t) * w->count, cudaMemcpyHostToDevice, s));
    int32_t cnt[2] = {0, w->count};
    B2P_CUDA(ctx, cudaMemcpyAsync(w->counters.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s));
    size_t sm = smem_bytes(w, sizeof(MT));
    ChunkFn<MT> fn = chunk_kernel<MT>(cfg.lc, cfg.lr);
    B2P_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    B2P_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, cfg.threads, sm));
    if (per_sm < 1) {
        ctx->err = "batch instance too large for one CTA's shared memory";
        return B2P_INVALID_ARGUMENT;
    }
    const int grid = ctx->sm_count * per_sm;
    BArgs a1 = make_args(w, p, vals_of<MT>(w, false), vals_of<MT>(w, true), w->active.p);
    BArgs a2 = make_args(w, p, vals_of<MT>(w, false), vals_of<MT>(w, true), w->active2.p);
    // one graph = two chunk launches with compaction (ping-pong active lists)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    B2P_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    fn<<<grid, cfg.threads, sm, s>>>(a1, cfg.chunk);
    k_batch_compact<<<1, 1024, 0, s>>>(w->ictrl.p, w->active.p, w->active2.p, w->counters.p);
    fn<<<grid, cfg.threads, sm, s>>>(a2, cfg.chunk);
    k_batch_compact<<<1, 1024, 0, s>>>(w->ictrl.p, w->active2.p, w->active.p, w->counters.p);
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) {
        ctx->err = std::string("batch graph capture: ") + cudaGetErrorString(ce);
        return B2P_EXECUTION_FAILED;
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        ctx->err = std::string("batch graph instantiate: ") + cudaGetErrorString(ce);
        return B2P_EXECUTION_FAILED;
    }
    int32_t* host_cnt = nullptr;
    B2P_CUDA(ctx, cudaMallocHost(&host_cnt, 2 * sizeof(int32_t)));
    const int64_t max_graphs = p->max_iterations / (2LL * cfg.chunk) + 3;
    int64_t graphs = 0;
    bool timed_out = false;
    const double tl = p->time_limit_s * 1000.0;
    cudaEventRecord(ctx->ev0, s);
    while (graphs < max_graphs) {
        B2P_CUDA(ctx, cudaGraphLaunch(exec, s));
        graphs++;
        B2P_CUDA(ctx, cudaMemcpyAsync(host_cnt, w->counters.p, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        B2P_CUDA(ctx, cudaStreamSynchronize(s));
        if (host_cnt[1] == 0) break;
        if (tl > 0 && now_ms() - t_start > tl) {
            timed_out = true;
            break;
        }
    }
    cudaEventRecord(ctx->ev1, s);
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    cudaFreeHost(host_cnt);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    ctx->launches += graphs * 4;
    float kms = 0;
    cudaEventElapsedTime(&kms, ctx->ev0, ctx->ev1);
    // results
    std::vector<InstCtrl> hc(w->count);
    B2P_CUDA(ctx, cudaMemcpyAsync(hc.data(), w->ictrl.p, sizeof(InstCtrl) * w->count, cudaMemcpyDeviceToHost, s));
    if (x_out || y_out) {
        DBuf<double> ox, oy;
        B2P_CUDA(ctx, ox.reserve(IN));
        B2P_CUDA(ctx, oy.reserve(IM));
        k_batch_unscale<double><<<std::min(w->count, ctx->sm_count * 8), 256, 0, s>>>(
            w->count, w->inst_mat.p, w->mat_m.p, w->mat_n.p, w->mat_row_off.p, w->mat_col_off.p, w->x_off.p, w->y_off.p,
            w->dr.p, w->dc.p, w->xt.p, w->yt.p, w->recenter ? w->xbar.p : nullptr, w->recenter ? w->ybar.p : nullptr,
            ox.p, oy.p);
        B2P_LAUNCH(ctx);
        ctx->launches += 1;
        if (x_out) B2P_CUDA(ctx, cudaMemcpyAsync(x_out, ox.p, sizeof(double) * IN, cudaMemcpyDeviceToHost, s));
        if (y_out) B2P_CUDA(ctx, cudaMemcpyAsync(y_out, oy.p, sizeof(double) * IM, cudaMemcpyDeviceToHost, s));
    }
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    int64_t tot_it = 0, opt = 0, maxit = 0;
    double worst = 0;
    for (int i = 0; i < w->count; ++i) {
        const InstCtrl& c = hc[i];
        int stt = c.done ? c.status : (timed_out ? B2P_STATUS_INTERRUPTED : B2P_STATUS_MAX_ITERATIONS);
        double kk = std::max(c.rel_p, std::max(c.rel_d, c.rel_g));
        if (status_out) status_out[i] = stt;
        if (iters_out) iters_out[i] = c.total;
        if (kkt_out) kkt_out[i] = kk;
        if (omega_out) omega_out[i] = c.omega;
        tot_it += c.total;
        maxit = std::max<int64_t>(maxit, c.total);
        opt += (stt == B2P_STATUS_OPTIMAL);
        worst = std::max(worst, kk);
    }
    if (sum) {
        sum->status = (opt == w->count) ? B2P_STATUS_OPTIMAL : (timed_out ? B2P_STATUS_INTERRUPTED : B2P_STATUS_MAX_ITERATIONS);
        sum->iterations = tot_it;   // sum over instances
        sum->restarts = maxit;      // longest instance
        sum->rel_kkt = worst;
        sum->kernel_time_ms = kms;
        sum->primal_weight = cfg.lc * 100 + cfg.lr;               // tuned lanes: column*100 + row
        sum->step_size = cfg.threads * 100000.0 + cfg.chunk;      // tuned threads*1e5 + chunk
    }
    return B2P_OK;
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
    // global CSR (block diagonal), host side
    std::vector<int64_t> row_off(nmat), col_off(nmat);
    int64_t tm = 0, tn = 0;
    for (int k = 0; k < nmat; ++k) {
        if (mat_m[k] <= 0 || mat_n[k] <= 0) {
            ctx->err = "b2p_batch_upload: empty matrix";
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
    std::vector<int32_t> grp(tm + 1), gci(nnz);
    int64_t rp_base = 0;
    grp[0] = 0;
    for (int k = 0; k < nmat; ++k) {
        const int32_t* rp = rowptr + rp_base;
        const int m = mat_m[k], n = mat_n[k];
        const int64_t e0 = mat_nnz_off[k], e1 = mat_nnz_off[k + 1];
        if (rp[0] != 0 || rp[m] != e1 - e0) {
            ctx->err = "b2p_batch_upload: matrix " + std::to_string(k) + " row pointers do not match its nnz";
            return B2P_INVALID_ARGUMENT;
        }
        for (int i = 0; i < m; ++i) {
            if (rp[i + 1] < rp[i]) {
                ctx->err = "b2p_batch_upload: decreasing row pointer";
                return B2P_INVALID_ARGUMENT;
            }
            grp[row_off[k] + i + 1] = (int32_t)(e0 + rp[i + 1]);
            int prev = -1;
            for (int e = rp[i]; e < rp[i + 1]; ++e) {
                int cidx = colidx[e0 + e];
                if (cidx < 0 || cidx >= n || cidx <= prev) {
                    ctx->err = "b2p_batch_upload: matrix " + std::to_string(k) + " row " + std::to_string(i) +
                               ": column indices out of range or not strictly ascending";
                    return B2P_INVALID_ARGUMENT;
                }
                prev = cidx;
                gci[e0 + e] = (int32_t)(cidx + col_off[k]);
            }
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
    for (auto* bf : {&w->rowptr}) B2P_CUDA(ctx, bf->reserve(tm + 1));
    B2P_CUDA(ctx, w->t_rowptr.reserve(tn + 1));
    for (auto* bf : {&w->colidx, &w->t_colidx}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->vals, &w->t_vals, &w->sv64, &w->stv64}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->sv32, &w->stv32}) B2P_CUDA(ctx, bf->reserve(nnz));
    for (auto* bf : {&w->dr, &w->pu}) B2P_CUDA(ctx, bf->reserve(tm));
    for (auto* bf : {&w->dc, &w->pv}) B2P_CUDA(ctx, bf->reserve(tn));
    for (auto* bf : {&w->mat_m, &w->mat_n}) B2P_CUDA(ctx, bf->reserve(nmat));
    for (auto* bf : {&w->mat_row_off, &w->mat_col_off}) B2P_CUDA(ctx, bf->reserve(nmat));
    B2P_CUDA(ctx, w->mat_eta.reserve(nmat));
    B2P_CUDA(ctx, w->inst_mat.reserve(count));
    for (auto* bf : {&w->x_off, &w->y_off}) B2P_CUDA(ctx, bf->reserve(count));
    for (auto* bf : {&w->c, &w->lb, &w->ub, &w->cs, &w->ls, &w->us, &w->x, &w->xa, &w->xt}) B2P_CUDA(ctx, bf->reserve(IN));
    for (auto* bf : {&w->b, &w->bs, &w->y, &w->ya, &w->yt}) B2P_CUDA(ctx, bf->reserve(IM));
    B2P_CUDA(ctx, w->is_eq.reserve(IM));
    for (auto* bf : {&w->bnorm, &w->cnorm}) B2P_CUDA(ctx, bf->reserve(count));
    B2P_CUDA(ctx, w->ictrl.reserve(count));
    for (auto* bf : {&w->active, &w->active2}) B2P_CUDA(ctx, bf->reserve(count));
    B2P_CUDA(ctx, w->counters.reserve(2));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->rowptr.p, grp.data(), sizeof(int32_t) * (tm + 1), cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->colidx.p, gci.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->vals.p, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_m.p, mat_m, sizeof(int32_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_n.p, mat_n, sizeof(int32_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_row_off.p, row_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->mat_col_off.p, col_off.data(), sizeof(int64_t) * nmat, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->inst_mat.p, inst_mat, sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->x_off.p, xoff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->y_off.p, yoff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->c.p, c, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->lb.p, lb, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->ub.p, ub, sizeof(double) * IN, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->b.p, b, sizeof(double) * IM, cudaMemcpyHostToDevice, s));
    B2P_CUDA(ctx, cudaMemcpyAsync(w->is_eq.p, is_eq, IM, cudaMemcpyHostToDevice, s));
    int st = build_transpose(ctx, (int)tm, (int)tn, nnz, w->rowptr.p, w->colidx.p, w->vals.p, w->t_rowptr.p,
                             w->t_colidx.p, w->t_vals.p);
    if (st) return st;
    // scaling + scaled values + step sizes (per matrix, FP64)
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
    B2P_LAUNCH(ctx);
    ctx->launches += 3;
    B2P_CUDA(ctx, cudaStreamSynchronize(s));
    return B2P_OK;
}

int b2p_batch_solve(void* p, const b2p_params* params, const double* x0, const double* y0, const double* omega0,
                    int32_t* status_out, int64_t* iters_out, double* kkt_out, double* omega_out, double* x_out,
                    double* y_out, b2p_result* summary) {
    Ctx* ctx = static_cast<Ctx*>(p);
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (!ctx->bw) {
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
    int st = pp->precision == B2P_FP64
                 ? batch_run<double>(ctx, ctx->bw, pp, x0, y0, omega0, status_out, iters_out, kkt_out, omega_out, x_out,
                                     y_out, summary)
                 : batch_run<float>(ctx, ctx->bw, pp, x0, y0, omega0, status_out, iters_out, kkt_out, omega_out, x_out,
                                    y_out, summary);
    if (summary) {
        summary->solve_time_ms = now_ms() - t0;
        summary->kernel_launches = ctx->launches - l0;
    }
    return st;
}

}  // extern "C"
