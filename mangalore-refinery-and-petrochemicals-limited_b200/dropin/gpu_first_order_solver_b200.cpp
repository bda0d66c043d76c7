// Drop-in GPU first-order solver for the reference BharatOpt library.
//
// Defines bharatopt::GPUFirstOrderSolver::{GPUFirstOrderSolver, solve} and
// bharatopt::FirstOrderLPSolver::{FirstOrderLPSolver, solve}
// (include/bharatopt/first_order_solver.hpp:89-113), replacing the versions in
// src/first_order_solver.cpp:292-319, which only ever ran the CPU solver.  That
// reference translation unit is compiled with
//   -DGPUFirstOrderSolver=RefGPUFirstOrderSolver -DFirstOrderLPSolver=RefFirstOrderLPSolver
// so its CPUFirstOrderSolver stays available and its GPU/dispatcher symbols do
// not clash with these.
//
// GPUFirstOrderSolver::solve keeps the reference's front end unchanged -- the
// same ModelValidator, PresolveEngine, closed-form answer for an empty reduced
// model, and standard form (first_order_solver.cpp:18-101, restated below
// because those steps are inline in the reference's solve) -- and hands the
// standard-form LP to libb2p through its C ABI.  Postsolve and the objective are
// again the reference's own (Postsolve::recover_solution,
// RevisedSimplex::recompute_original_objective).
//
// Engine selection: by default the reference engine (B2P_ENGINE_REFERENCE), which
// reproduces CPUFirstOrderSolver's iterates, status and iteration count with the
// options' max_iterations / check_frequency / tolerances / step sizes.  The
// restarted Halpern engine is chosen by bharatopt_b200_set_engine() or by the
// environment (B2P_ENGINE=halpern, B2P_PRECISION=fp32|fp64, B2P_EPS=<rel KKT>).
// There is no CPU fallback: without a usable GPU the result is NUMERICAL_FAILURE
// with a message saying so (the router's own DualRevisedSimplex fallback,
// src/execution_router.cpp:277-298, stays the caller's business).
//
// Direct setup (bharatopt_b200_set_setup(1) or B2P_SETUP=direct): instead of the
// validator + presolve + standard form above (90 + 174 ms of host time at 800k
// nonzeros, more than a whole GPU solve of the block-angular LP), one pass over the
// model's rows, split over the host's cores, writes the standard form's CSR
// directly -- G rows negated, a ranged row [rhs, range_upper] as two <= rows (an
// equality when the ends coincide; the reference's path keeps only its lower end,
// first_order_solver.cpp:83-99), duplicate terms summed -- checking bounds and
// coefficients on the way (NaN -> NUMERICAL_FAILURE, lb > ub -> INFEASIBLE_DETECTED).
// The engine's transpose, scaling and layouts are built on the device as always;
// the answer needs no postsolve, and the duals are mapped back to the model's rows
// (negated for G rows, upper minus lower for ranged rows).
#include <bharatopt/first_order_solver.hpp>
#include <bharatopt/model_validator.hpp>
#include <bharatopt/presolve.hpp>
#include <bharatopt/revised_simplex.hpp>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/b2p.h"
#include "b2p_dropin.hpp"

namespace {

std::mutex g_mutex;
void* g_ctx = nullptr;
bool g_have_override = false;
b2p_params g_override;
int g_setup = -1;  // -1: from the environment, 0: reference front end, 1: direct

bool direct_setup() {
    if (g_setup >= 0) return g_setup == 1;
    const char* e = std::getenv("B2P_SETUP");
    return e && std::strcmp(e, "direct") == 0;
}

// Standard form of `model` written directly (see the file header).  first_row / kind give
// the standard rows of each model row; status 0 ok, 1 NaN found, 2 lb > ub.
struct DirectForm {
    int m = 0, n = 0;
    std::vector<int32_t> rowptr, colidx;
    std::vector<double> vals, b, c, lb, ub;
    std::vector<uint8_t> is_eq;
    std::vector<int32_t> first_row;   // per model row: its first standard row
    std::vector<int8_t> kind;         // per model row: 0 L, 1 E, 2 G, 3 ranged (two rows), 4 ranged equality,
                                      // 5 ranged with only its upper end, 6 with only its lower end, 7 none
    int status = 0;
    std::string why;
};

void build_direct(const bharatopt::LPModel& model, DirectForm& f) {
    using namespace bharatopt;
    const size_t n = model.num_variables(), m = model.num_constraints();
    f.n = (int)n;
    const double sense = model.sense() == ObjectiveSense::MINIMIZE ? 1.0 : -1.0;
    f.c.resize(n);
    f.lb.resize(n);
    f.ub.resize(n);
    for (size_t j = 0; j < n; ++j) {
        const Variable& v = model.get_variable((index_t)j);
        if (std::isnan(v.obj_coeff) || std::isnan(v.lower_bound) || std::isnan(v.upper_bound)) {
            f.status = 1;
            f.why = "NaN cost or bound of variable " + v.name;
            return;
        }
        if (v.lower_bound > v.upper_bound) {
            f.status = 2;
            f.why = "contradictory bounds of variable " + v.name;
            return;
        }
        f.c[j] = sense * v.obj_coeff;
        f.lb[j] = v.lower_bound;
        f.ub[j] = v.upper_bound;
    }
    // row kinds and the number of standard rows each model row becomes
    f.kind.resize(m);
    f.first_row.resize(m + 1);
    f.first_row[0] = 0;
    for (size_t i = 0; i < m; ++i) {
        const Constraint& con = model.get_constraint((index_t)i);
        int8_t k = con.sense == ConstraintSense::LESS_EQUAL ? 0 : con.sense == ConstraintSense::EQUAL ? 1
                 : con.sense == ConstraintSense::GREATER_EQUAL ? 2 : 3;
        if (k == 3) {
            const bool lo_fin = std::isfinite(con.rhs), hi_fin = std::isfinite(con.range_upper);
            if (con.rhs == con.range_upper) k = 4;
            else if (!lo_fin && hi_fin) k = 5;
            else if (lo_fin && !hi_fin) k = 6;
            else if (!lo_fin && !hi_fin) k = 7;
        }
        f.kind[i] = k;
        f.first_row[i + 1] = f.first_row[i] + (k == 3 ? 2 : k == 7 ? 0 : 1);
    }
    const size_t ms = (size_t)f.first_row[m];
    f.m = (int)ms;
    f.b.assign(ms, 0.0);
    f.is_eq.assign(ms, 0);
    // rows in parallel: each worker sorts and merges its rows' terms into a local CSR piece
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t T = std::max<size_t>(1, std::min<size_t>(hw, m / 2048 + 1));
    struct Piece {
        std::vector<int32_t> len, col;
        std::vector<double> val;
        int status = 0;
        std::string why;
    };
    std::vector<Piece> piece(T);
    auto work = [&](size_t t) {
        Piece& P = piece[t];
        const size_t i0 = m * t / T, i1 = m * (t + 1) / T;
        std::vector<std::pair<int32_t, double>> e;
        for (size_t i = i0; i < i1; ++i) {
            const Constraint& con = model.get_constraint((index_t)i);
            e.clear();
            for (const auto& term : con.terms) {
                if (std::isnan(term.second) || term.first < 0 || (size_t)term.first >= n) {
                    P.status = 1;
                    P.why = "bad term in row " + con.name;
                    return;
                }
                e.push_back({(int32_t)term.first, term.second});
            }
            std::sort(e.begin(), e.end(), [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                return a.first < b.first;
            });
            size_t w = 0;
            for (size_t q = 0; q < e.size(); ++q) {
                if (w > 0 && e[w - 1].first == e[q].first) e[w - 1].second += e[q].second;
                else e[w++] = e[q];
            }
            const int8_t k = f.kind[i];
            const int copies = k == 3 ? 2 : k == 7 ? 0 : 1;
            for (int r = 0; r < copies; ++r) {
                // sign of this standard row: G rows, the lower end of a ranged row negated
                const bool neg = k == 2 || (k == 3 && r == 1) || k == 6;
                const size_t row = (size_t)f.first_row[i] + r;
                double rhs = con.rhs;
                if (k == 3 && r == 0) rhs = con.range_upper;
                if (k == 5) rhs = con.range_upper;
                f.b[row] = neg ? -rhs : rhs;
                f.is_eq[row] = (k == 1 || k == 4) ? 1 : 0;
                P.len.push_back((int32_t)w);
                for (size_t q = 0; q < w; ++q) {
                    P.col.push_back(e[q].first);
                    P.val.push_back(neg ? -e[q].second : e[q].second);
                }
            }
        }
    };
    std::vector<std::thread> th;
    for (size_t t = 1; t < T; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    for (auto& P : piece)
        if (P.status) {
            f.status = P.status;
            f.why = P.why;
            return;
        }
    f.rowptr.assign(ms + 1, 0);
    size_t r = 0, z = 0;
    for (auto& P : piece) {
        for (int32_t l : P.len) {
            f.rowptr[r + 1] = f.rowptr[r] + l;
            ++r;
        }
        z += P.col.size();
    }
    f.colidx.reserve(z);
    f.vals.reserve(z);
    for (auto& P : piece) {
        f.colidx.insert(f.colidx.end(), P.col.begin(), P.col.end());
        f.vals.insert(f.vals.end(), P.val.begin(), P.val.end());
    }
}

void* solver_context() {
    if (!g_ctx) {
        void* c = nullptr;
        if (b2p_ctx_create(0, &c) == B2P_OK) g_ctx = c;
    }
    return g_ctx;
}

// Reference-engine parameters from FirstOrderSolverOptions (first_order_solver.hpp:29-38),
// or the Halpern engine when selected.
b2p_params engine_params(const bharatopt::FirstOrderSolverOptions& o) {
    b2p_params p;
    if (g_have_override) {
        p = g_override;
    } else {
        b2p_params_default(&p);
        const char* e = std::getenv("B2P_ENGINE");
        if (e && std::strcmp(e, "halpern") == 0) {
            p.engine = B2P_ENGINE_HALPERN;
            const char* pr = std::getenv("B2P_PRECISION");
            p.precision = (pr && std::strcmp(pr, "fp64") == 0) ? B2P_FP64 : B2P_FP32;
            const char* eps = std::getenv("B2P_EPS");
            if (eps) p.eps_rel_kkt = std::atof(eps);
        }
    }
    p.max_iterations = (int64_t)o.max_iterations;
    if (p.engine == B2P_ENGINE_REFERENCE) {
        p.feasibility_tolerance = o.feasibility_tolerance;
        p.primal_step_size = o.primal_step_size;
        p.dual_step_size = o.dual_step_size;
        p.adaptive_step_size = o.adaptive_step_size ? 1 : 0;
        p.check_frequency = (int64_t)o.check_frequency;
    }
    return p;
}

}  // namespace

extern "C" void bharatopt_b200_set_setup(int direct) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_setup = direct < 0 ? -1 : (direct ? 1 : 0);
}

extern "C" void bharatopt_b200_set_engine(const b2p_params* params) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (params) {
        g_override = *params;
        g_have_override = true;
    } else {
        g_have_override = false;
    }
}

namespace bharatopt {

GPUFirstOrderSolver::GPUFirstOrderSolver(FirstOrderSolverOptions options) : options_(options) {}

namespace {

// The direct-setup path of GPUFirstOrderSolver::solve (see the file header).
FirstOrderSolverResult solve_direct(const LPModel& model, const FirstOrderSolverOptions& options,
                                    std::chrono::high_resolution_clock::time_point start_time) {
    FirstOrderSolverResult result;
    DirectForm f;
    build_direct(model, f);
    const double setup_ms =
        std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - start_time).count();
    if (f.status == 1) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        result.message = "Model validation failed before First-Order LP Solver: " + f.why;
        return result;
    }
    if (f.status == 2) {
        result.status = FirstOrderSolverStatus::INFEASIBLE_DETECTED;
        result.message = "Infeasible: " + f.why;
        return result;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    void* ctx = solver_context();
    if (!ctx) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        b2p_device_info_t info;
        b2p_device_info(0, &info);
        result.message = std::string("B200 first-order engine unavailable: ") + info.status_message;
        return result;
    }
    b2p_params params = engine_params(options);
    if (params.engine == B2P_ENGINE_REFERENCE) {  // direct setup runs the Halpern engine
        params.engine = B2P_ENGINE_HALPERN;
        params.precision = B2P_FP64;
    }
    int st = b2p_upload_lp(ctx, f.m, f.n, (int64_t)f.vals.size(), f.rowptr.data(), f.colidx.data(), f.vals.data(),
                           f.b.data(), f.c.data(), f.lb.data(), f.ub.data(), f.is_eq.data());
    b2p_result r;
    std::memset(&r, 0, sizeof(r));
    std::vector<real_t> x(f.n, 0.0), y(f.m, 0.0);
    if (st == B2P_OK) st = b2p_solve(ctx, &params, nullptr, nullptr, &r, x.data(), y.data());
    if (st != B2P_OK) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        result.message = std::string("B200 first-order engine failed: ") + b2p_last_error(ctx);
        return result;
    }
    switch (r.status) {
        case B2P_STATUS_OPTIMAL: result.status = FirstOrderSolverStatus::OPTIMAL; break;
        case B2P_STATUS_MAX_ITERATIONS: result.status = FirstOrderSolverStatus::MAX_ITERATIONS; break;
        case B2P_STATUS_INFEASIBLE_DETECTED: result.status = FirstOrderSolverStatus::INFEASIBLE_DETECTED; break;
        case B2P_STATUS_UNBOUNDED_DETECTED: result.status = FirstOrderSolverStatus::UNBOUNDED_DETECTED; break;
        case B2P_STATUS_INTERRUPTED: result.status = FirstOrderSolverStatus::INTERRUPTED; break;
        default: result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE; break;
    }
    result.message = "B200 Halpern engine, direct setup (" + std::to_string(setup_ms) + " ms host setup)";
    // duals per model row: negated for G rows, upper minus lower for a two-sided ranged row
    std::vector<real_t> yd(model.num_constraints(), 0.0);
    for (size_t i = 0; i < yd.size(); ++i) {
        const int32_t q = f.first_row[i];
        switch (f.kind[i]) {
            case 0: case 1: case 4: case 5: yd[i] = y[q]; break;
            case 2: case 6: yd[i] = -y[q]; break;
            case 3: yd[i] = y[q] - y[q + 1]; break;
            default: break;
        }
    }
    result.primal_solution = x;
    result.dual_solution = yd;
    RevisedSimplex verifier;
    result.objective_value = verifier.recompute_original_objective(model, result.primal_solution);
    result.stats.primal_objective = result.objective_value;
    result.stats.dual_objective = r.dual_objective;
    result.stats.iterations = (size_t)r.iterations;
    result.stats.primal_residual = r.rel_primal_residual;
    result.stats.dual_residual = r.rel_dual_residual;
    result.stats.kernel_time_ms = r.kernel_time_ms;
    result.stats.transfer_time_ms = r.transfer_time_ms;
    result.stats.solve_time_ms =
        std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - start_time).count();
    return result;
}

}  // namespace

FirstOrderSolverResult GPUFirstOrderSolver::solve(const LPModel& model) {
    FirstOrderSolverResult result;
    auto start_time = std::chrono::high_resolution_clock::now();
    if (direct_setup()) return solve_direct(model, options_, start_time);

    // 1. validation (first_order_solver.cpp:19-25)
    ModelValidator validator;
    if (!validator.validate(model).is_valid()) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        result.message = "Model validation failed before First-Order LP Solver.";
        return result;
    }
    // 2. presolve (:28-34)
    PresolveEngine presolver;
    PresolveResult pre = presolver.presolve(model);
    if (pre.status == PresolveStatus::INFEASIBLE) {
        result.status = FirstOrderSolverStatus::INFEASIBLE_DETECTED;
        result.message = "Presolve detected infeasibility.";
        return result;
    }
    const LPModel& work = pre.reduced_model;
    const size_t m = work.num_constraints(), n = work.num_variables();
    const real_t sense_mult = (work.sense() == ObjectiveSense::MINIMIZE) ? 1.0 : -1.0;

    // 3. no constraints or no variables left: bound optimisation (:42-66)
    if (m == 0 || n == 0) {
        std::vector<real_t> x_red(n, 0.0);
        for (size_t j = 0; j < n; ++j) {
            const auto& var = work.get_variable(static_cast<index_t>(j));
            const real_t cj = var.obj_coeff * sense_mult;
            const real_t lj = var.lower_bound, uj = var.upper_bound;
            if (cj > 1e-12) x_red[j] = (lj > -BHARATOPT_INFINITY) ? lj : 0.0;
            else if (cj < -1e-12) x_red[j] = (uj < BHARATOPT_INFINITY) ? uj : 0.0;
            else x_red[j] = bharatopt::clamp(0.0, (lj > -BHARATOPT_INFINITY) ? lj : -1e9, (uj < BHARATOPT_INFINITY) ? uj : 1e9);
        }
        result.primal_solution = pre.postsolve.recover_solution(x_red);
        result.status = FirstOrderSolverStatus::OPTIMAL;
        RevisedSimplex verifier;
        result.objective_value = verifier.recompute_original_objective(model, result.primal_solution);
        result.stats.primal_objective = result.objective_value;
        result.message = "LP model solved via bound optimization & presolve postsolve.";
        return result;
    }

    // 4. standard form A x (<= | =) b, >= rows negated (:68-101)
    COOMatrix coo(m, n);
    std::vector<real_t> b(m, 0.0), c(n, 0.0), lb(n, 0.0), ub(n, BHARATOPT_INFINITY);
    std::vector<uint8_t> is_eq(m, 0);
    for (size_t j = 0; j < n; ++j) {
        const auto& var = work.get_variable(static_cast<index_t>(j));
        c[j] = var.obj_coeff * sense_mult;
        lb[j] = var.lower_bound;
        ub[j] = var.upper_bound;
    }
    for (size_t i = 0; i < m; ++i) {
        const auto& cons = work.get_constraint(static_cast<index_t>(i));
        real_t rhs = cons.rhs, mult = 1.0;
        if (cons.sense == ConstraintSense::GREATER_EQUAL) {
            rhs = -rhs;
            mult = -1.0;
        } else if (cons.sense == ConstraintSense::EQUAL) {
            is_eq[i] = 1;
        }
        b[i] = rhs;
        for (const auto& term : cons.terms) coo.add_entry(static_cast<index_t>(i), term.first, term.second * mult);
    }
    CSRMatrix A = CSRMatrix::from_coo(coo);

    // 5. the GPU engine
    std::lock_guard<std::mutex> lock(g_mutex);
    void* ctx = solver_context();
    if (!ctx) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        b2p_device_info_t info;
        b2p_device_info(0, &info);
        result.message = std::string("B200 first-order engine unavailable: ") + info.status_message;
        return result;
    }
    int st = b2p_upload_lp(ctx, (int)m, (int)n, (int64_t)A.nnz(), A.row_offsets().data(), A.col_indices().data(),
                           A.values().data(), b.data(), c.data(), lb.data(), ub.data(), is_eq.data());
    b2p_params params = engine_params(options_);
    b2p_result r;
    std::memset(&r, 0, sizeof(r));
    std::vector<real_t> x(n, 0.0), y(m, 0.0);
    if (st == B2P_OK) st = b2p_solve(ctx, &params, nullptr, nullptr, &r, x.data(), y.data());
    if (st != B2P_OK) {
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        result.message = std::string("B200 first-order engine failed: ") + b2p_last_error(ctx);
        return result;
    }
    result.stats.constraint_violation = r.constraint_violation;
    result.stats.bound_violation = r.bound_violation;
    if (params.engine == B2P_ENGINE_REFERENCE && r.status == B2P_STATUS_NUMERICAL_FAILURE) {
        // the reference returns at the failing check without a solution (:232-236)
        result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
        result.message = "Numerical failure: exploded iterate detected during PDHG iterations.";
        return result;
    }
    auto end_time = std::chrono::high_resolution_clock::now();
    result.stats.solve_time_ms = std::chrono::duration<double, std::milli>(end_time - start_time).count();
    result.stats.kernel_time_ms = r.kernel_time_ms;
    result.stats.transfer_time_ms = r.transfer_time_ms;
    result.stats.iterations = (size_t)r.iterations;
    result.stats.primal_residual = r.rel_primal_residual;
    result.stats.dual_residual = r.rel_dual_residual;
    result.stats.dual_objective = r.dual_objective;
    switch (r.status) {
        case B2P_STATUS_OPTIMAL:
            result.status = FirstOrderSolverStatus::OPTIMAL;
            result.message = "PDHG/PDLP-style first-order solver converged to OPTIMAL solution.";
            break;
        case B2P_STATUS_MAX_ITERATIONS:
            result.status = FirstOrderSolverStatus::MAX_ITERATIONS;
            result.message = "PDHG/PDLP-style first-order solver reached maximum iteration limit.";
            break;
        case B2P_STATUS_INTERRUPTED:
            result.status = FirstOrderSolverStatus::INTERRUPTED;
            result.message = "B200 first-order engine stopped at its time limit.";
            break;
        case B2P_STATUS_INFEASIBLE_DETECTED:
            result.status = FirstOrderSolverStatus::INFEASIBLE_DETECTED;
            result.message = "B200 first-order engine found a dual ray certifying primal infeasibility.";
            break;
        case B2P_STATUS_UNBOUNDED_DETECTED:
            result.status = FirstOrderSolverStatus::UNBOUNDED_DETECTED;
            result.message = "B200 first-order engine found a primal ray certifying unboundedness.";
            break;
        default:
            result.status = FirstOrderSolverStatus::NUMERICAL_FAILURE;
            result.message = "B200 first-order engine reported a numerical failure.";
            break;
    }
    result.message += (params.engine == B2P_ENGINE_REFERENCE) ? " [B200 reference engine]" : " [B200 Halpern engine]";
    // 6. postsolve, duals, objective on the original model (:282-287)
    result.primal_solution = pre.postsolve.recover_solution(x);
    result.dual_solution = y;
    RevisedSimplex verifier;
    result.objective_value = verifier.recompute_original_objective(model, result.primal_solution);
    result.stats.primal_objective = result.objective_value;
    return result;
}

FirstOrderLPSolver::FirstOrderLPSolver(FirstOrderSolverOptions options) : options_(options) {}

// first_order_solver.cpp:311-319: GPU_FIRST_ORDER -> the B200 engine; CPU_FIRST_ORDER -> the
// reference's own CPUFirstOrderSolver, exactly as requested by the caller.
FirstOrderSolverResult FirstOrderLPSolver::solve(const LPModel& model) {
    if (options_.backend_type == FirstOrderBackendType::GPU_FIRST_ORDER) {
        GPUFirstOrderSolver solver(options_);
        return solver.solve(model);
    }
    CPUFirstOrderSolver solver(options_);
    return solver.solve(model);
}

}  // namespace bharatopt
