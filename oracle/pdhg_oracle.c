/*
 * ORACLE — test infrastructure only. Never linked into, or called by, the
 * product library. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it, and only as the checker.
 *
 * Plain-C restatement of the reference PDHG loop, CPUFirstOrderSolver::solve
 * (src/first_order_solver.cpp), for an LP already in the reference's standard
 * form  A x (<= | =) b,  lb <= x <= ub  (rows flagged by is_eq).  Statement
 * order and arithmetic order follow the reference line by line so that, built
 * with the same compiler flags (no FMA contraction), the iterates are
 * bit-identical to the compiled reference:
 *   steps tau/sigma ........ first_order_solver.cpp:103-128
 *   x0 / y0 / buffers ...... :130-151
 *   A^T y (row scatter) .... :163  -> sparse_matrix.cpp:175-185
 *   primal step + x_sum .... :165-175
 *   extrapolation .......... :177-180
 *   A x_hat (row gather) ... :183  -> sparse_matrix.cpp:153-163
 *   dual step .............. :185-192
 *   x_prev = x ............. :194
 *   convergence check ...... :197-246
 *   final x / x_avg pick ... :249-279
 * Parity of this restatement is pinned against the compiled reference
 * (oracle/_ref/libbharatopt_ref.so) by tests/test_oracle.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int status;            /* 0 OPTIMAL, 1 MAX_ITERATIONS, 2 NUMERICAL_FAILURE */
    long iterations;       /* loop counter at exit */
    double constraint_violation;
    double bound_violation;
    double max_primal_delta;
    double max_dual_delta;
    int used_average;      /* 1 if x_final is the ergodic average */
} OracleRefResult;

static double clampd(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

/* sparse_matrix.cpp:153-163 */
void oracle_spmv(int m, const int* rowptr, const int* colidx, const double* vals, const double* x, double* y) {
    for (int i = 0; i < m; ++i) {
        double sum = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) sum += vals[k] * x[colidx[k]];
        y[i] = sum;
    }
}

/* sparse_matrix.cpp:175-185 */
void oracle_spmv_t(int m, int n, const int* rowptr, const int* colidx, const double* vals, const double* y, double* w) {
    for (int j = 0; j < n; ++j) w[j] = 0.0;
    for (int i = 0; i < m; ++i) {
        double yi = y[i];
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) w[colidx[k]] += vals[k] * yi;
    }
}

/* std::max(a, b) is (a < b) ? b : a, so a NaN violation never replaces the running maximum. */
static double max_row_violation(int m, const double* ax, const double* b, const unsigned char* is_eq) {
    double mv = 0.0;
    for (int i = 0; i < m; ++i) {
        double d = ax[i] - b[i];
        double v = (!is_eq[i]) ? ((0.0 < d) ? d : 0.0) : fabs(d);
        mv = (mv < v) ? v : mv;
    }
    return mv;
}

int oracle_ref_pdhg(int m, int n, const int* rowptr, const int* colidx, const double* vals,
                    const double* b, const double* c, const double* lb, const double* ub,
                    const unsigned char* is_eq, long max_iterations, long check_frequency,
                    double feas_tol, int adaptive, double primal_step, double dual_step,
                    double* x_final, double* x_last, double* y_last, double* x_sum_out,
                    OracleRefResult* res) {
    double* col_sums = calloc((size_t)n, sizeof(double));
    double* row_sums = calloc((size_t)m, sizeof(double));
    double* tau = malloc((size_t)n * sizeof(double));
    double* sigma = malloc((size_t)m * sizeof(double));
    double* x = malloc((size_t)n * sizeof(double));
    double* y = calloc((size_t)m, sizeof(double));
    double* x_hat = calloc((size_t)n, sizeof(double));
    double* x_prev = malloc((size_t)n * sizeof(double));
    double* at_y = calloc((size_t)n, sizeof(double));
    double* a_xhat = calloc((size_t)m, sizeof(double));
    double* x_sum = calloc((size_t)n, sizeof(double));
    double* ax = malloc((size_t)m * sizeof(double));
    double* x_avg = malloc((size_t)n * sizeof(double));
    const double INF = INFINITY;

    for (int i = 0; i < m; ++i)
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            double a = fabs(vals[k]);
            row_sums[i] += a;
            col_sums[colidx[k]] += a;
        }
    for (int j = 0; j < n; ++j) tau[j] = primal_step;
    for (int i = 0; i < m; ++i) sigma[i] = dual_step;
    if (adaptive) {
        for (int j = 0; j < n; ++j) tau[j] = (col_sums[j] > 1e-12) ? (0.95 / col_sums[j]) : 1.0;
        for (int i = 0; i < m; ++i) sigma[i] = (row_sums[i] > 1e-12) ? (0.95 / row_sums[i]) : 1.0;
    }
    for (int j = 0; j < n; ++j) {
        double target = 0.0;
        if (lb[j] > -INF && ub[j] < INF) target = 0.5 * (lb[j] + ub[j]);
        else if (lb[j] > -INF) target = lb[j];
        else if (ub[j] < INF) target = ub[j];
        x[j] = clampd(target, lb[j], ub[j]);
        x_prev[j] = x[j];
    }

    long avg_count = 0, iter = 0;
    int converged = 0;
    long check_freq = check_frequency < 100 ? check_frequency : 100;
    double max_primal_delta = 0.0, max_dual_delta = 0.0;
    memset(res, 0, sizeof(*res));
    res->status = 1;

    while (iter < max_iterations) {
        iter++;
        oracle_spmv_t(m, n, rowptr, colidx, vals, y, at_y);
        max_primal_delta = 0.0;
        for (int j = 0; j < n; ++j) {
            double grad = c[j] + at_y[j];
            double next_x = x[j] - tau[j] * grad;
            double new_x = clampd(next_x, lb[j], ub[j]);
            double d = fabs(new_x - x[j]);
            if (d > max_primal_delta) max_primal_delta = d;
            x[j] = new_x;
            x_sum[j] += x[j];
        }
        avg_count++;
        for (int j = 0; j < n; ++j) x_hat[j] = 2.0 * x[j] - x_prev[j];
        oracle_spmv(m, rowptr, colidx, vals, x_hat, a_xhat);
        max_dual_delta = 0.0;
        for (int i = 0; i < m; ++i) {
            double next_y = y[i] + sigma[i] * (a_xhat[i] - b[i]);
            double new_y = (!is_eq[i]) ? (0.0 > next_y ? 0.0 : next_y) : next_y;
            double d = fabs(new_y - y[i]);
            if (d > max_dual_delta) max_dual_delta = d;
            y[i] = new_y;
        }
        memcpy(x_prev, x, (size_t)n * sizeof(double));

        if (iter % check_freq == 0 || iter == max_iterations) {
            oracle_spmv(m, rowptr, colidx, vals, x, ax);
            double max_viol = max_row_violation(m, ax, b, is_eq);
            double max_bound_viol = 0.0;
            for (int j = 0; j < n; ++j) {
                if (x[j] < lb[j] - 1e-12 && lb[j] - x[j] > max_bound_viol) max_bound_viol = lb[j] - x[j];
                if (x[j] > ub[j] + 1e-12 && x[j] - ub[j] > max_bound_viol) max_bound_viol = x[j] - ub[j];
            }
            for (int j = 0; j < n; ++j) x_avg[j] = clampd(x_sum[j] / (double)avg_count, lb[j], ub[j]);
            oracle_spmv(m, rowptr, colidx, vals, x_avg, ax);
            double avg_viol = max_row_violation(m, ax, b, is_eq);
            /* std::min(max_viol, avg_viol) returns the first argument unless the second is smaller */
            double best_viol = (avg_viol < max_viol) ? avg_viol : max_viol;
            res->constraint_violation = best_viol;
            res->bound_violation = max_bound_viol;
            if (isnan(best_viol) || best_viol > 1e15) {
                res->status = 2;
                res->iterations = iter;
                goto done;
            }
            int is_feasible = (best_viol <= feas_tol && max_bound_viol <= feas_tol);
            int is_stationary = (max_primal_delta <= 1e-7 && max_dual_delta <= 1e-7);
            if (is_feasible && is_stationary && iter >= 100) { converged = 1; break; }
        }
    }
    res->iterations = iter;
    res->status = converged ? 0 : 1;
    if (avg_count > 0) {
        for (int j = 0; j < n; ++j) x_avg[j] = clampd(x_sum[j] / (double)avg_count, lb[j], ub[j]);
    } else {
        memcpy(x_avg, x, (size_t)n * sizeof(double));
    }
    oracle_spmv(m, rowptr, colidx, vals, x_avg, ax);
    {
        double avg_viol = max_row_violation(m, ax, b, is_eq);
        int use_avg = (!converged) && (avg_viol <= res->constraint_violation);
        res->used_average = use_avg;
        memcpy(x_final, use_avg ? x_avg : x, (size_t)n * sizeof(double));
    }
done:
    res->max_primal_delta = max_primal_delta;
    res->max_dual_delta = max_dual_delta;
    if (x_last) memcpy(x_last, x, (size_t)n * sizeof(double));
    if (y_last) memcpy(y_last, y, (size_t)m * sizeof(double));
    if (x_sum_out) memcpy(x_sum_out, x_sum, (size_t)n * sizeof(double));
    free(col_sums); free(row_sums); free(tau); free(sigma); free(x); free(y); free(x_hat);
    free(x_prev); free(at_y); free(a_xhat); free(x_sum); free(ax); free(x_avg);
    return res->status;
}
