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
#include <bharatopt/first_order_solver.hpp>
#include <bharatopt/model_validator.hpp>
#include <bharatopt/presolve.hpp>
#include <bharatopt/revised_simplex.hpp>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/b2p.h"
#include "b2p_dropin.hpp"

namespace {

std::mutex g_mutex;
void* g_ctx = nullptr;
bool g_have_override = false;
b2p_params g_override;

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

FirstOrderSolverResult GPUFirstOrderSolver::solve(const LPModel& model) {
    FirstOrderSolverResult result;
    auto start_time = std::chrono::high_resolution_clock::now();

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
