/*
 * b2p.h -- C ABI of the B200 PDHG LP engine (libb2p.so).
 *
 * This is the drop-in boundary for the reference BharatOpt first-order LP
 * path.  The reference's C++ entry points bind to it as follows (reference
 * file:line of each interface replaced):
 *
 *   GpuBackend::initialize / device_info   include/bharatopt/gpu_backend.hpp:173-177
 *        -> b2p_device_info, b2p_ctx_create
 *   GpuBackend::spmv / spmv_with_cpu_comparison  gpu_backend.hpp:180-190
 *        -> b2p_spmv
 *   GpuBackend::vector_add/_sub/_scale, axpy     gpu_backend.hpp:193-216
 *        -> b2p_vector_op
 *   GpuBackend::dot_product / norm2              gpu_backend.hpp:218-227
 *        -> b2p_dot, b2p_norm2
 *   GPUFirstOrderSolver::solve                   include/bharatopt/first_order_solver.hpp:89-98
 *   (src/first_order_solver.cpp:295-306)
 *        -> b2p_upload_lp + b2p_solve  (after the reference's own validation,
 *           presolve and standard form, src/first_order_solver.cpp:18-101)
 *   FirstOrderSolverStats / Result / Status      first_order_solver.hpp:15-60
 *        -> b2p_result, B2P_STATUS_*
 *
 * Entry points with no reference counterpart (new engine capabilities):
 *   b2p_batch_*  -- thousands of independent LPs in one persistent launch
 *   b2p_mlp_*    -- learned warm start (BF16 tensor-core MLP)
 *
 * Conventions: plain pointers and sizes; every pointer argument is HOST
 * memory unless its name ends in _dev.  Every function returns an int status
 * (B2P_OK on success) and never throws.  A context owns one CUDA stream and
 * all device buffers it allocates; it is not re-entrant (one host thread per
 * context at a time).  There is no CPU fallback: without a usable GPU every
 * compute entry point returns B2P_GPU_UNAVAILABLE.
 */
#ifndef B2P_H
#define B2P_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- call status; 0..5 have the meaning of bharatopt::GPUStatus
 *      (include/bharatopt/gpu_backend.hpp:15-22) ---- */
#define B2P_OK                  0
#define B2P_GPU_UNAVAILABLE     1
#define B2P_GPU_UNINITIALIZED   2
#define B2P_OUT_OF_MEMORY       3
#define B2P_INVALID_ARGUMENT    4
#define B2P_EXECUTION_FAILED    5
#define B2P_NO_LP               6   /* solve before upload */
#define B2P_TIMEOUT             7   /* a bounded device wait or the time limit ran out */

/* ---- solver outcome; same ordinals as bharatopt::FirstOrderSolverStatus
 *      (include/bharatopt/first_order_solver.hpp:15-22) ---- */
#define B2P_STATUS_OPTIMAL              0
#define B2P_STATUS_MAX_ITERATIONS       1
#define B2P_STATUS_NUMERICAL_FAILURE    2
#define B2P_STATUS_INFEASIBLE_DETECTED  3
#define B2P_STATUS_UNBOUNDED_DETECTED   4
#define B2P_STATUS_INTERRUPTED          5

/* ---- engines ---- */
#define B2P_ENGINE_REFERENCE  0  /* the reference PDHG, iterate-for-iterate (FP64 only) */
#define B2P_ENGINE_HALPERN    1  /* restarted Halpern PDHG, scaled, rel-KKT termination */

#define B2P_FP64  0
#define B2P_FP32  1              /* FP32 vectors + SpMV, FP64 reductions / scaling / KKT */

typedef struct {
    int    is_available;
    char   device_name[128];
    size_t total_memory_bytes;
    size_t free_memory_bytes;
    int    compute_capability_major;
    int    compute_capability_minor;
    int    multiprocessor_count;
    int    l2_cache_bytes;
    char   status_message[256];
} b2p_device_info_t;

/* Host-observed phase times in milliseconds (GpuTimingResult,
 * include/bharatopt/gpu_backend.hpp:34-41); kernel time from CUDA events. */
typedef struct {
    double h2d_time_ms;
    double kernel_time_ms;
    double d2h_time_ms;
    double sync_time_ms;
    double total_gpu_time_ms;
} b2p_timing_t;

typedef struct {
    int     engine;                 /* B2P_ENGINE_* */
    int     precision;              /* B2P_FP64 / B2P_FP32 (Halpern engine only) */
    int64_t max_iterations;         /* default 50000 (first_order_solver.hpp:30) */
    /* reference engine (FirstOrderSolverOptions, first_order_solver.hpp:29-38) */
    double  feasibility_tolerance;  /* 1e-7 */
    double  primal_step_size;       /* 0.01, used when adaptive_step_size == 0 */
    double  dual_step_size;         /* 0.01 */
    int     adaptive_step_size;     /* 1 */
    int64_t check_frequency;        /* 100 (clamped to <= 100 like the reference) */
    /* Halpern engine */
    double  eps_rel_kkt;            /* 1e-6: primal, dual and gap all within eps relative */
    int     check_every;            /* 64 iterations per chunk (restart / KKT cadence) */
    int     ruiz_iterations;        /* 10 */
    double  reflection;             /* 1.0 = reflected Halpern */
    double  restart_sufficient;     /* 0.2 */
    double  restart_necessary;      /* 0.8 */
    double  restart_artificial;     /* 0.36 */
    double  primal_weight;          /* 0 = ||c||/||b|| of the scaled LP */
    double  step_safety;            /* 0.998 / ||A||_2 */
    int     refinement_rounds;      /* FP64 iterative refinement: at each restart the LP is re-centred on the
                                       current point with residuals b - A x, c + A^T y computed from the
                                       FP64 matrix.  -1 = on for FP32 / off for FP64 (default), 0 = off,
                                       > 0 = on */
    double  time_limit_s;           /* 0 = none */
    int     lanes_per_row;          /* Halpern engine iteration kernels: 0 = autotuned; 1,2,4,8,16,32 =
                                       CSR kernel with that many lanes per row; -1 = SELL kernel, 32-row
                                       slices; -2 = the same with gather windows in shared memory;
                                       -3 / -4 = SELL kernel, 16- / 8-row slices (2 / 4 lanes per row) */
    /* Halpern and batched engines */
    double  eps_objective;          /* 0 = off (default).  > 0: OPTIMAL also needs the answer's objective
                                       c.x within eps_objective * max(1, |c.x|) of the optimum, judged by
                                       the FP64 bound max(c.x - d(y), sum_i |y_i| viol_i(x)): d(y) is the
                                       dual objective (a lower bound on the optimum when the reduced costs
                                       are absorbed by the bounds), the sum bounds how far below the
                                       optimum an infeasible x can reach to first order */
    double  eps_infeasible;         /* 1e-8: PDLP-style certificates from the fixed-point displacement
                                       T(z) - z at the restart checks (every check in the single-LP
                                       engine, every fourth in the batched one).  Dual ray dy (primal
                                       infeasible): its ray
                                       objective -b.dy + sum_j min(a_j l_j, a_j u_j), a = A^T dy, is > 0
                                       and the violations of a on unbounded sides are <= eps_infeasible
                                       times it -> B2P_STATUS_INFEASIBLE_DETECTED.  Primal ray dx (dual
                                       infeasible): c.dx < 0 and the violations of A dx and of the bound
                                       recession cone are <= eps_infeasible |c.dx| ->
                                       B2P_STATUS_UNBOUNDED_DETECTED.  0 = off */
} b2p_params;

typedef struct {
    int     status;                 /* B2P_STATUS_* */
    int64_t iterations;
    int64_t restarts;
    double  primal_objective;       /* c.x of the standard-form LP */
    double  dual_objective;
    double  rel_primal_residual;    /* FP64, original (unscaled) LP */
    double  rel_dual_residual;
    double  rel_gap;
    double  rel_kkt;                /* max of the three */
    double  constraint_violation;   /* max |viol| (reference engine: FirstOrderSolverStats) */
    double  bound_violation;
    double  max_primal_delta;
    double  max_dual_delta;
    int     used_average;           /* reference engine picked the ergodic average */
    int     refinement_rounds_done;
    double  primal_weight;
    double  step_size;
    double  solve_time_ms;          /* host wall time of b2p_solve */
    double  kernel_time_ms;         /* CUDA-event time of the iteration loop */
    double  transfer_time_ms;       /* host<->device copies inside b2p_solve */
    int64_t kernel_launches;        /* kernels this call launched (graph nodes counted) */
} b2p_result;

/* ---- device, context ---- */
int  b2p_device_info(int device, b2p_device_info_t* out);
int  b2p_ctx_create(int device, void** ctx_out);
int  b2p_ctx_destroy(void* ctx);
const char* b2p_last_error(void* ctx);      /* message of the last failed call (never null) */
/* Run all of this context's work on the caller's CUDA stream (cudaStream_t passed
 * as void*; null restores the context's own stream).  Lets a caller order and
 * time the engine's kernels with its own events. */
int  b2p_ctx_set_stream(void* ctx, void* stream);
void b2p_params_default(b2p_params* p);

/* ---- GpuBackend primitives (host buffers; FP64 CSR with int32 indices) ---- */
int b2p_spmv(void* ctx, int m, int n, const int32_t* rowptr, const int32_t* colidx, const double* vals,
             const double* x, double* y, b2p_timing_t* timing);
int b2p_spmv_t(void* ctx, int m, int n, const int32_t* rowptr, const int32_t* colidx, const double* vals,
               const double* y, double* w, b2p_timing_t* timing);
#define B2P_VEC_ADD   0   /* out = a + b          */
#define B2P_VEC_SUB   1   /* out = a - b          */
#define B2P_VEC_SCALE 2   /* out = alpha * a      */
#define B2P_VEC_AXPY  3   /* out = alpha * a + b  */
int b2p_vector_op(void* ctx, int op, size_t n, double alpha, const double* a, const double* b, double* out,
                  b2p_timing_t* timing);
int b2p_dot(void* ctx, size_t n, const double* a, const double* b, double* out, b2p_timing_t* timing);
int b2p_norm2(void* ctx, size_t n, const double* a, double* out, b2p_timing_t* timing);

/* Allocation-free dot product.  No counterpart in the reference: it exists for
 * callers that cannot let a library allocate device memory -- code recording a
 * CUDA graph (cudaMalloc is not allowed while a stream is being captured) or an
 * application that owns all device memory through its own pool.  The caller
 * passes DEVICE pointers: a_dev, b_dev (n doubles each) and out_dev (1 double,
 * receives a.b).  Work is queued on `stream` (a cudaStream_t; null = legacy
 * default stream) and the call returns without synchronising.  No context is
 * needed and nothing is allocated: the partial sums go to a fixed 32 KiB array
 * in the library's device memory, which every GPU that loads the library keeps
 * until the process exits.
 *   - n may be at most B2P_DOT_NOALLOC_MAX_N; larger n returns B2P_TOO_LARGE
 *     before anything is launched.
 *   - The first call on a device looks the array's address up (set-up); make
 *     that first call before any stream capture on that device.
 *   - Every call shares the array (each call overwrites all it reads), so two
 *     calls that can run at the same time on the GPU -- on different streams or
 *     from different threads -- race; serialise them on one stream.
 *   - A CUDA error left pending by earlier work is returned as this call's
 *     status and nothing is launched.  The set-up is cached per device for the
 *     life of the process: cudaDeviceReset is not supported. */
#define B2P_TOO_LARGE           8
#define B2P_DOT_NOALLOC_MAX_N   8388608
int b2p_dot_noalloc(const double* a_dev, const double* b_dev, size_t n, double* out_dev, void* stream);

/* ---- single LP ----
 * Standard form (src/first_order_solver.cpp:68-101): minimise c.x subject to
 * (A x)_i <= b_i where is_eq[i] == 0, (A x)_i == b_i where is_eq[i] == 1, and
 * lb <= x <= ub (entries may be +-inf).  A is CSR with int32 indices, column
 * indices strictly ascending within each row (CSRMatrix::is_valid,
 * src/sparse_matrix.cpp:187-207).  The context keeps one uploaded LP. */
int b2p_upload_lp(void* ctx, int m, int n, int64_t nnz, const int32_t* rowptr, const int32_t* colidx,
                  const double* vals, const double* b, const double* c, const double* lb, const double* ub,
                  const uint8_t* is_eq);
/* x0 (n) / y0 (m) optional warm start (Halpern engine); x_out (n) / y_out (m) optional. */
int b2p_solve(void* ctx, const b2p_params* params, const double* x0, const double* y0, b2p_result* result,
              double* x_out, double* y_out);

/* ---- MPS -> device ingest (replaces MpsParser::parse_file,
 *      include/bharatopt/mps_parser.hpp:40-48, src/mps_parser.cpp:140-531, on the way
 *      to the engine).  The file is read on the host in one pass straight into CSR, with
 *      the reference parser's semantics (sections, markers, first RHS / RANGES / BOUNDS
 *      vector, range table, bound types, objective offset); b2p_upload_mps uploads its
 *      standard form: G rows negated, a ranged row [lo, hi] as a.x <= hi and
 *      -a.x <= -lo (an equality when lo == hi).  Host code only: reading needs no GPU. */
typedef struct b2p_mps b2p_mps;
/* Reads `path`; on failure returns B2P_INVALID_ARGUMENT with the reason and line in err. */
int  b2p_mps_read(const char* path, b2p_mps** out, char* err, size_t errlen);
void b2p_mps_free(b2p_mps* mps);
/* Sizes: m rows (objective excluded), n columns, nnz; objective sense and offset; the
 * standard form's rows and nonzeros.  Any pointer may be null. */
int  b2p_mps_dims(const b2p_mps* mps, int* m, int* n, int64_t* nnz, int* maximize, double* obj_offset, int* std_m,
                  int64_t* std_nnz);
/* The model as read: CSR of the rows (column indices ascending), row_type 'L' / 'G' / 'E',
 * ranged flag, rhs (a ranged row's lower end), range upper end; per column cost, bounds and
 * kind (0 continuous, 1 integer, 2 binary).  Any pointer may be null. */
int  b2p_mps_model(const b2p_mps* mps, int32_t* rowptr, int32_t* colidx, double* vals, char* row_type,
                   uint8_t* ranged, double* rhs, double* range_upper, double* obj, double* lb, double* ub,
                   uint8_t* col_type);
/* The standard form (std_m rows) in b2p_upload_lp's layout; c is negated for maximisation. */
int  b2p_mps_standard_form(const b2p_mps* mps, int32_t* rowptr, int32_t* colidx, double* vals, double* b,
                           double* c, double* lb, double* ub, uint8_t* is_eq);
/* b2p_upload_lp of the standard form. */
int  b2p_upload_mps(void* ctx, const b2p_mps* mps);

/* Per-kernel timing of the Halpern iteration on the uploaded LP, after a
 * b2p_solve with the same params: `reps` plain iterations launched one kernel
 * at a time between CUDA events on the context stream.  Returns the mean
 * duration of the primal kernel (A^T y + primal step) and of the dual kernel
 * (A xh + dual step) and the algorithmic bytes each moves per launch (every
 * matrix entry, row pointer and vector element read or written once). */
int b2p_kernel_timing(void* ctx, const b2p_params* params, int reps, double* primal_ms, double* dual_ms,
                      double* primal_bytes, double* dual_bytes);

/* ---- batch of independent LPs (no reference counterpart) ----
 * `nmat` constraint matrices in concatenated CSR (mat_rowptr_off[k] indexes
 * rowptr, mat_nnz_off[k] indexes colidx/vals; rowptr entries are local to their
 * matrix).  `count` instances each name a matrix (inst_mat) and bring their own
 * b (m of that matrix), c, lb, ub (n) and is_eq, concatenated in instance order.
 * Many instances may share one matrix (parametric families). */
int b2p_batch_upload(void* ctx, int nmat, const int32_t* mat_m, const int32_t* mat_n,
                     const int64_t* mat_nnz_off, const int32_t* rowptr, const int32_t* colidx, const double* vals,
                     int count, const int32_t* inst_mat, const double* b, const double* c, const double* lb,
                     const double* ub, const uint8_t* is_eq);
/* Solve all instances with the Halpern engine.  x0/y0 optional warm starts
 * (concatenated like c / b), omega0 optional per-instance primal weights.
 * Outputs (optional): per-instance status, iterations, rel KKT and final primal
 * weight; concatenated x, y.  The summary reports the autotuned kernel shape:
 * step_size = CTA size * 1e5 + chunk length (iterations per persistent launch),
 * used_average = 10 * instances per CTA (2: the paired form, batches whose
 * instances share one matrix) + SELL entries per lane load.  The shape is tuned
 * once per batch signature and cached in the file B2P_AUTOTUNE_CACHE (default
 * ~/.cache/b2p_autotune.txt); B2P_BATCH_SHAPE="threads,w,ni" pins it. */
int b2p_batch_solve(void* ctx, const b2p_params* params, const double* x0, const double* y0, const double* omega0,
                    int32_t* status_out, int64_t* iters_out, double* kkt_out, double* omega_out, double* x_out,
                    double* y_out, b2p_result* summary);

/* Per-instance objectives of the last batched solve (count each; any pointer may
 * be null): the primal objective c.x, the dual objective d(y) -- a valid lower
 * bound on the optimum when every column is boxed, which is what a
 * branch-and-bound search prunes on (the reference prunes on the node LP's
 * objective, src/branch_and_bound.cpp:517-537) -- and the FP64 bound on the
 * relative objective error of the answer (see b2p_params.eps_objective). */
int b2p_batch_objectives(void* ctx, double* pobj_out, double* dobj_out, double* obj_err_out);

/* Active-instance trace of the last batched solve (no reference counterpart): after
 * every replay of the persistent-kernel graph (two chunk launches and their
 * compactions) the host time in ms since the solve's first launch and the number of
 * instances still running; a learned solve's cold fallback continues the trace.
 * Writes up to `capacity` points and the total in *count. */
int b2p_batch_trace(void* ctx, int capacity, int* count, double* t_ms, int32_t* active);

/* ---- learned warm start: MLP in -> h -> h -> out, GELU, BF16 weights and
 *      activations, FP32 accumulation on the tcgen05 tensor cores ---- */
int b2p_mlp_create(void* ctx, int in_dim, int hidden, int out_dim, uint64_t seed);
/* One pass of Adam over N samples (X: N x in_dim, Y: N x out_dim, FP32 row-major,
 * host).  loss_out (optional) receives the mean squared error of the epoch. */
int b2p_mlp_train_epoch(void* ctx, const float* X, const float* Y, int N, int batch, float lr, float* loss_out);
int b2p_mlp_infer(void* ctx, const float* X, int N, float* Y_out);
/* All parameters as one FP32 vector: W1 [hidden x in], b1 [hidden], W2 [hidden x
 * hidden], b2 [hidden], W3 [out x hidden], b3 [out] (row-major). */
int b2p_mlp_get_params(void* ctx, float* flat);
int b2p_mlp_set_params(void* ctx, const float* flat);
/* Mean-squared-error loss of one batch and its gradient (flat layout as above),
 * computed by the same tensor-core forward / backward the training step uses. */
int b2p_mlp_gradient(void* ctx, const float* X, const float* Y, int N, float* loss_out, float* grad_flat);
/* Training set on the device from the answers of the last b2p_batch_solve: the
 * inputs are the instances' parameter vectors (count x in_dim, FP32 host, one per
 * instance of the batch), the targets their [x (n), y (m), log(final primal
 * weight)] in the original space, so out_dim must be n + m + 1 and every
 * instance of the batch must share that shape.  Sets the normalisation
 * (per-column means; one scale per block x / y / weight).  No solution data
 * crosses to the host.  No reference counterpart (the reference has no learned
 * component). */
int b2p_mlp_dataset_from_batch(void* ctx, const float* features, int count);
/* `epochs` passes of Adam over the device training set, reshuffled every epoch
 * (seeded), learning rate cosine-annealed from lr_start to lr_end.  loss_out
 * (optional): mean squared error of the last epoch, in normalised units. */
int b2p_mlp_train(void* ctx, int epochs, int batch, float lr_start, float lr_end, uint64_t seed, float* loss_out);
/* Normalisation used by the dataset and the learned solve: in_mean/in_std
 * [in_dim], out_mean/out_std [out_dim] (with the weights, a trained model). */
int b2p_mlp_get_normalization(void* ctx, float* in_mean, float* in_std, float* out_mean, float* out_std);
int b2p_mlp_set_normalization(void* ctx, const float* in_mean, const float* in_std, const float* out_mean,
                              const float* out_std);
/* Learned warm start, all on the device: the MLP maps every instance's parameter
 * vector (features: count x in_dim, FP32 host) to x0, y0 and a primal weight, the
 * batch is solved from there (params->precision; default FP32 + re-centring), and
 * with `fallback` != 0 every instance the warm-started run did not solve (a
 * numerical failure of a bad prediction) is solved again from the cold start with
 * the iterations left of max_iterations: the count continues, so warm + cold stay
 * within the cap.  Outputs as b2p_batch_solve, plus warm_used_out[i] = 1 when
 * instance i's answer came from the warm start; the iteration count of a
 * fallen-back instance includes its warm-started run.
 * summary->refinement_rounds_done = number of instances that fell back.  Replaces
 * the reference's cold-start-only GPUFirstOrderSolver::solve
 * (src/first_order_solver.cpp:295-306) for parametric families. */
int b2p_batch_solve_learned(void* ctx, const b2p_params* params, const float* features, int fallback,
                            int32_t* status_out, int64_t* iters_out, double* kkt_out, uint8_t* warm_used_out,
                            double* x_out, double* y_out, b2p_result* summary);
/* Raw BF16 GEMM on the tensor cores, for tests: C(MxN, fp32) = op(A) op(B),
 * A is M x K (trans_a = 0) or K x M (trans_a = 1) bf16 row-major, B is K x N
 * (trans_b = 0) or N x K (trans_b = 1).  Host buffers (bf16 as uint16). */
int b2p_gemm_bf16(void* ctx, int M, int N, int K, const uint16_t* A, int trans_a, const uint16_t* B, int trans_b,
                  float* C);

#ifdef __cplusplus
}
#endif
#endif /* B2P_H */
