// Oracle shim (test infrastructure only; never linked into the product).
//
// extern "C" wrappers over the reference BharatOpt classes so that the Python
// tests and the CPU-baseline leg of bench.py can call the reference's own code
// through ctypes:
//   ref_fo_solve      -> CPUFirstOrderSolver::solve   (src/first_order_solver.cpp:14-290)
//   ref_sf_*          -> PresolveEngine::presolve     (src/presolve.cpp:157-515) followed by the
//                        standard-form construction of src/first_order_solver.cpp:68-101 and
//                        CSRMatrix::from_coo (src/sparse_matrix.cpp:59-111)
//   ref_spmv/_t       -> CSRMatrix::multiply / multiply_transpose (src/sparse_matrix.cpp:153-185)
//   ref_verify        -> SolutionVerifier::verify     (src/solution_verifier.cpp:42-204)
//   ref_mps_*         -> MpsParser::parse_file        (src/mps_parser.cpp:140-531), the LPModel it
//                        builds read out row by row
#include <bharatopt/first_order_solver.hpp>
#include <bharatopt/mps_parser.hpp>
#include <bharatopt/presolve.hpp>
#include <bharatopt/solution_verifier.hpp>
#include <bharatopt/sparse_matrix.hpp>
#include <bharatopt/lp_model.hpp>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace bharatopt;

extern "C" {

// Row-wise description of an original (not yet standardised) LP.
struct RefLP {
    int m, n;
    const int* rowptr;        // m+1
    const int* colidx;        // nnz
    const double* vals;       // nnz
    const int* sense;         // m: 0 <=, 1 =, 2 >=, 3 ranged
    const double* rhs;        // m
    const double* range_upper;// m (may be null)
    const double* obj;        // n
    const double* lb;         // n
    const double* ub;         // n
    int maximize;
    double obj_offset;
};

struct RefFOResult {
    int status;               // FirstOrderSolverStatus ordinal
    long iterations;
    double objective;
    double constraint_violation;
    double bound_violation;
    double solve_time_ms;
    long n_primal;
    long n_dual;
};

struct RefVerifyResult {
    int verified;
    double objective_recomputed;
    double max_constraint_violation;
    double max_lower_bound_violation;
    double max_upper_bound_violation;
    long violated_constraints;
    long violated_bounds;
};
}

static LPModel build_model(const RefLP* lp) {
    LPModel model("oracle_lp");
    model.set_sense(lp->maximize ? ObjectiveSense::MAXIMIZE : ObjectiveSense::MINIMIZE);
    model.set_obj_offset(lp->obj_offset);
    for (int j = 0; j < lp->n; ++j) {
        model.add_variable("x" + std::to_string(j), lp->lb[j], lp->ub[j], lp->obj[j]);
    }
    static const ConstraintSense senses[4] = {ConstraintSense::LESS_EQUAL, ConstraintSense::EQUAL,
                                              ConstraintSense::GREATER_EQUAL, ConstraintSense::RANGED};
    std::vector<std::pair<index_t, real_t>> terms;
    for (int i = 0; i < lp->m; ++i) {
        terms.clear();
        for (int k = lp->rowptr[i]; k < lp->rowptr[i + 1]; ++k) terms.push_back({lp->colidx[k], lp->vals[k]});
        model.add_constraint("r" + std::to_string(i), terms, senses[lp->sense[i]], lp->rhs[i],
                             lp->range_upper ? lp->range_upper[i] : 0.0);
    }
    return model;
}

extern "C" {

int ref_fo_solve(const RefLP* lp, long max_iterations, long check_frequency, double feas_tol,
                 int adaptive_step, double primal_step, double dual_step,
                 RefFOResult* out, double* x_out, long x_cap, double* y_out, long y_cap) {
    LPModel model = build_model(lp);
    FirstOrderSolverOptions opts;
    opts.max_iterations = static_cast<size_t>(max_iterations);
    opts.check_frequency = static_cast<size_t>(check_frequency);
    opts.feasibility_tolerance = feas_tol;
    opts.adaptive_step_size = adaptive_step != 0;
    opts.primal_step_size = primal_step;
    opts.dual_step_size = dual_step;
    opts.backend_type = FirstOrderBackendType::CPU_FIRST_ORDER;
    CPUFirstOrderSolver solver(opts);
    FirstOrderSolverResult r = solver.solve(model);
    out->status = static_cast<int>(r.status);
    out->iterations = static_cast<long>(r.stats.iterations);
    out->objective = r.objective_value;
    out->constraint_violation = r.stats.constraint_violation;
    out->bound_violation = r.stats.bound_violation;
    out->solve_time_ms = r.stats.solve_time_ms;
    out->n_primal = static_cast<long>(r.primal_solution.size());
    out->n_dual = static_cast<long>(r.dual_solution.size());
    if (x_out) for (long j = 0; j < (long)r.primal_solution.size() && j < x_cap; ++j) x_out[j] = r.primal_solution[j];
    if (y_out) for (long i = 0; i < (long)r.dual_solution.size() && i < y_cap; ++i) y_out[i] = r.dual_solution[i];
    return 0;
}

// ---- presolve + standard form, as CPUFirstOrderSolver::solve sees the LP ----
struct RefSF {
    LPModel original;
    PresolveResult pre;
    int status;  // 0 ok, 1 presolve infeasible, 2 empty (m==0||n==0)
    int m, n;
    std::vector<index_t> rowptr, colidx;
    std::vector<real_t> vals, b, c, lb, ub;
    std::vector<unsigned char> is_eq;
};

void* ref_sf_create(const RefLP* lp) {
    RefSF* h = new RefSF();
    h->original = build_model(lp);
    PresolveEngine presolver;
    h->pre = presolver.presolve(h->original);
    h->status = 0;
    h->m = h->n = 0;
    if (h->pre.status == PresolveStatus::INFEASIBLE) { h->status = 1; return h; }
    const LPModel& w = h->pre.reduced_model;
    size_t m = w.num_constraints(), n = w.num_variables();
    h->m = (int)m; h->n = (int)n;
    if (m == 0 || n == 0) { h->status = 2; return h; }
    real_t sense_mult = (w.sense() == ObjectiveSense::MINIMIZE) ? 1.0 : -1.0;
    COOMatrix coo(m, n);
    h->b.assign(m, 0.0); h->c.assign(n, 0.0); h->lb.assign(n, 0.0); h->ub.assign(n, 0.0);
    h->is_eq.assign(m, 0);
    for (size_t j = 0; j < n; ++j) {
        const auto& v = w.get_variable((index_t)j);
        h->c[j] = v.obj_coeff * sense_mult;
        h->lb[j] = v.lower_bound;
        h->ub[j] = v.upper_bound;
    }
    for (size_t i = 0; i < m; ++i) {
        const auto& cons = w.get_constraint((index_t)i);
        real_t rhs = cons.rhs, mult = 1.0;
        if (cons.sense == ConstraintSense::GREATER_EQUAL) { rhs = -rhs; mult = -1.0; }
        else if (cons.sense == ConstraintSense::EQUAL) { h->is_eq[i] = 1; }
        h->b[i] = rhs;
        for (const auto& t : cons.terms) coo.add_entry((index_t)i, t.first, t.second * mult);
    }
    CSRMatrix A = CSRMatrix::from_coo(coo);
    h->rowptr = A.row_offsets();
    h->colidx = A.col_indices();
    h->vals = A.values();
    return h;
}

void ref_sf_dims(void* hv, int* status, int* m, int* n, int* nnz) {
    RefSF* h = (RefSF*)hv;
    *status = h->status; *m = h->m; *n = h->n; *nnz = (int)h->vals.size();
}

void ref_sf_copy(void* hv, int* rowptr, int* colidx, double* vals, double* b, double* c,
                 double* lb, double* ub, unsigned char* is_eq) {
    RefSF* h = (RefSF*)hv;
    std::memcpy(rowptr, h->rowptr.data(), h->rowptr.size() * sizeof(int));
    std::memcpy(colidx, h->colidx.data(), h->colidx.size() * sizeof(int));
    std::memcpy(vals, h->vals.data(), h->vals.size() * sizeof(double));
    std::memcpy(b, h->b.data(), h->b.size() * sizeof(double));
    std::memcpy(c, h->c.data(), h->c.size() * sizeof(double));
    std::memcpy(lb, h->lb.data(), h->lb.size() * sizeof(double));
    std::memcpy(ub, h->ub.data(), h->ub.size() * sizeof(double));
    std::memcpy(is_eq, h->is_eq.data(), h->is_eq.size());
}

// Postsolve::recover_solution (src/presolve.cpp:51-78) + objective on the original model.
double ref_sf_recover(void* hv, const double* x_red, long n_red, double* x_orig) {
    RefSF* h = (RefSF*)hv;
    std::vector<real_t> xr(x_red, x_red + n_red);
    std::vector<real_t> xo = h->pre.postsolve.recover_solution(xr);
    for (size_t j = 0; j < xo.size(); ++j) x_orig[j] = xo[j];
    real_t obj = h->original.obj_offset();
    for (size_t j = 0; j < xo.size(); ++j) obj += h->original.get_variable((index_t)j).obj_coeff * xo[j];
    return obj;
}

void ref_sf_free(void* hv) { delete (RefSF*)hv; }

// ---- SpMV on the reference CSRMatrix ----
static CSRMatrix make_csr(int m, int n, const int* rowptr, const int* colidx, const double* vals) {
    int nnz = rowptr[m];
    return CSRMatrix((size_t)m, (size_t)n, std::vector<index_t>(rowptr, rowptr + m + 1),
                     std::vector<index_t>(colidx, colidx + nnz), std::vector<real_t>(vals, vals + nnz));
}

int ref_spmv(int m, int n, const int* rowptr, const int* colidx, const double* vals,
             const double* x, double* y) {
    try { make_csr(m, n, rowptr, colidx, vals).multiply(x, y); } catch (...) { return -1; }
    return 0;
}

int ref_spmv_t(int m, int n, const int* rowptr, const int* colidx, const double* vals,
               const double* y, double* w) {
    try { make_csr(m, n, rowptr, colidx, vals).multiply_transpose(y, w); } catch (...) { return -1; }
    return 0;
}

int ref_verify(const RefLP* lp, const double* x, double feas_tol, double reported_obj, int check_obj,
               RefVerifyResult* out) {
    LPModel model = build_model(lp);
    VerificationOptions opts;
    opts.feasibility_tolerance = feas_tol;
    opts.check_objective = check_obj != 0;
    SolutionVerifier v;
    std::vector<real_t> cand(x, x + lp->n);
    VerificationResult r = check_obj ? v.verify(model, cand, reported_obj, opts) : v.verify(model, cand, opts);
    out->verified = r.verified ? 1 : 0;
    out->objective_recomputed = r.objective_recomputed;
    out->max_constraint_violation = r.maximum_constraint_violation;
    out->max_lower_bound_violation = r.maximum_lower_bound_violation;
    out->max_upper_bound_violation = r.maximum_upper_bound_violation;
    out->violated_constraints = (long)r.violated_constraint_count;
    out->violated_bounds = (long)r.violated_bound_count;
    return 0;
}

// ---- MPS through the reference's parser ----
struct RefMps {
    MpsParseResult res;
};

// Parses `path`; returns a handle (null on a parse failure, with the message in err).
void* ref_mps_parse(const char* path, char* err, int errlen) {
    MpsParser parser;
    RefMps* h = new RefMps();
    h->res = parser.parse_file(path);
    if (h->res.status != MpsParseStatus::SUCCESS) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", h->res.error_message.c_str());
        delete h;
        return nullptr;
    }
    return h;
}

void ref_mps_dims(void* hv, int* m, int* n, int* nnz, int* maximize, double* obj_offset) {
    const LPModel& md = ((RefMps*)hv)->res.model;
    *m = (int)md.num_constraints();
    *n = (int)md.num_variables();
    size_t z = 0;
    for (size_t i = 0; i < md.num_constraints(); ++i) z += md.get_constraint((index_t)i).terms.size();
    *nnz = (int)z;
    *maximize = md.sense() == ObjectiveSense::MAXIMIZE ? 1 : 0;
    *obj_offset = md.obj_offset();
}

// Rows as CSR in each row's term order; sense 0 <=, 1 =, 2 >=, 3 ranged; variable type
// 0 continuous, 1 integer, 2 binary.
void ref_mps_copy(void* hv, int* rowptr, int* colidx, double* vals, int* sense, double* rhs, double* range_upper,
                  double* obj, double* lb, double* ub, int* vtype) {
    const LPModel& md = ((RefMps*)hv)->res.model;
    rowptr[0] = 0;
    for (size_t i = 0; i < md.num_constraints(); ++i) {
        const Constraint& c = md.get_constraint((index_t)i);
        int p = rowptr[i];
        for (const auto& t : c.terms) {
            colidx[p] = t.first;
            vals[p++] = t.second;
        }
        rowptr[i + 1] = p;
        sense[i] = c.sense == ConstraintSense::LESS_EQUAL ? 0 : c.sense == ConstraintSense::EQUAL ? 1
                 : c.sense == ConstraintSense::GREATER_EQUAL ? 2 : 3;
        rhs[i] = c.rhs;
        range_upper[i] = c.range_upper;
    }
    for (size_t j = 0; j < md.num_variables(); ++j) {
        const Variable& v = md.get_variable((index_t)j);
        obj[j] = v.obj_coeff;
        lb[j] = v.lower_bound;
        ub[j] = v.upper_bound;
        vtype[j] = v.type == VariableType::CONTINUOUS ? 0 : v.type == VariableType::INTEGER ? 1 : 2;
    }
}

void ref_mps_free(void* hv) { delete (RefMps*)hv; }

}  // extern "C"
