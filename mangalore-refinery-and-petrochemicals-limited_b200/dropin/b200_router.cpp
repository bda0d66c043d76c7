// B200-calibrated cost estimator and adaptive router (see b200_router.hpp).
#include "b200_router.hpp"

#include <algorithm>
#include <string>

#include <bharatopt/gpu_backend.hpp>
#include <bharatopt/milp_foundation.hpp>

namespace bharatopt {

namespace {

const char* kModelVersion = "b200-calibrated-v1";

CostEstimate first_order(const char* variant, double total_ms, double compute_ms, double transfer_ms,
                         GpuExecutionStatus gs, const std::string& profile) {
    CostEstimate e;
    e.solver_name = "FirstOrderLP";
    e.solver_variant = variant;
    e.predicted_total_time_ms = total_ms;
    e.predicted_compute_time_ms = compute_ms;
    e.predicted_transfer_time_ms = transfer_ms;
    e.gpu_execution_status = gs;
    e.model_version = kModelVersion;
    e.hardware_profile = profile;
    e.extrapolation_message = "B200 calibration (measured per-nonzero costs; typical iteration count)";
    return e;
}

}  // namespace

CostEstimate B200CostEstimator::estimate(const WorkloadFeatures& f, BenchmarkSolverType solver) const {
    const double nnz = static_cast<double>(f.nnz);
    const double prologue = cal_.host_prologue_ms_per_nnz * nnz;
    if (solver == BenchmarkSolverType::CPU_FIRST_ORDER) {
        const double iter = cal_.cpu_pdhg_iter_ms + cal_.cpu_pdhg_iter_ms_per_nnz * nnz;
        const double compute = cal_.cpu_pdhg_iterations * iter;
        return first_order("CPU_PDHG", prologue + compute, compute, 0.0, GpuExecutionStatus::INVALID,
                           "host CPU, one core");
    }
    if (solver == BenchmarkSolverType::GPU_FIRST_ORDER) {
        if (!(f.gpu_available && GpuBackend::instance().is_available())) {
            // no device: the drop-in has no host fallback, so the GPU path cannot run
            CostEstimate e = first_order("GPU_PDHG", 1e30, 1e30, 0.0, GpuExecutionStatus::GPU_UNAVAILABLE,
                                         "no usable B200");
            e.prediction_valid = false;
            e.validity_status = ValidityStatus::INVALID;
            return e;
        }
        const double setup = cal_.gpu_setup_ms + cal_.gpu_setup_ms_per_nnz * nnz;
        const double compute = cal_.gpu_iterations * (cal_.gpu_iter_ms + cal_.gpu_iter_ms_per_nnz * nnz);
        return first_order("GPU_PDHG", prologue + setup + compute, compute, setup, GpuExecutionStatus::NATIVE_GPU,
                           f.gpu_name.empty() ? std::string("B200") : f.gpu_name);
    }
    return simplex_.estimate(f, solver);
}

std::vector<CostEstimate> B200CostEstimator::estimate_all(const WorkloadFeatures& f) const {
    return {estimate(f, BenchmarkSolverType::REVISED_SIMPLEX), estimate(f, BenchmarkSolverType::DUAL_REVISED_SIMPLEX),
            estimate(f, BenchmarkSolverType::CPU_FIRST_ORDER), estimate(f, BenchmarkSolverType::GPU_FIRST_ORDER)};
}

B200ExecutionRouter::B200ExecutionRouter(RoutingConfiguration config, std::shared_ptr<ICostEstimator> estimator)
    : ExecutionRouter(config, estimator ? estimator : std::make_shared<B200CostEstimator>()) {}

RoutingDecision B200ExecutionRouter::decide(const LPModel& model, const WorkloadFeatures& features,
                                            const std::vector<CostEstimate>& estimates) {
    RoutingDecision d = ExecutionRouter::decide(model, features, estimates);
    // forced modes and MILP models keep the reference's decision
    if (config().routing_mode != RoutingMode::ADAPTIVE || d.selected_solver == BenchmarkSolverType::BRANCH_AND_BOUND)
        return d;
    double rev = 1e300, dual = 1e300, cpu_fo = 1e300, gpu_fo = 1e300;
    for (const auto& e : estimates) {
        if (e.solver_name == "RevisedSimplex") rev = e.predicted_total_time_ms;
        else if (e.solver_name == "DualRevisedSimplex") dual = e.predicted_total_time_ms;
        else if (e.solver_variant == "CPU_PDHG") cpu_fo = e.predicted_total_time_ms;
        else if (e.solver_variant == "GPU_PDHG" && e.prediction_valid) gpu_fo = e.predicted_total_time_ms;
    }
    const double best_cpu = std::min({rev, dual, cpu_fo});
    const bool gpu_usable = features.gpu_available && features.cuda_available && config().gpu_allowed;
    d.predicted_cpu_cost_ms = best_cpu;
    d.predicted_gpu_cost_ms = gpu_fo;
    d.estimator_version = kModelVersion;
    const std::string costs = "(predicted GPU PDHG " + std::to_string(gpu_fo) + " ms vs best CPU " +
                              std::to_string(best_cpu) + " ms, margin " +
                              std::to_string(config().min_gpu_speedup_margin_ms) + " ms)";
    if (gpu_usable && gpu_fo + config().min_gpu_speedup_margin_ms < best_cpu) {
        d.selected_solver = BenchmarkSolverType::GPU_FIRST_ORDER;
        d.solver_name = "FirstOrderLP";
        d.solver_variant = "GPU_PDHG";
        d.execution_device = "GPU";
        d.selected_predicted_cost_ms = gpu_fo;
        d.routing_reason = "B200_CALIBRATED_GPU_SELECTED: " + costs;
        return d;
    }
    // the cheapest CPU solver of the calibrated estimates
    if (best_cpu == rev) {
        d.selected_solver = BenchmarkSolverType::REVISED_SIMPLEX;
        d.solver_name = "RevisedSimplex";
        d.solver_variant = "CPU_Revised_Simplex";
    } else if (best_cpu == dual) {
        d.selected_solver = BenchmarkSolverType::DUAL_REVISED_SIMPLEX;
        d.solver_name = "DualRevisedSimplex";
        d.solver_variant = "CPU_Dual_Simplex";
    } else {
        d.selected_solver = BenchmarkSolverType::CPU_FIRST_ORDER;
        d.solver_name = "FirstOrderLP";
        d.solver_variant = "CPU_PDHG";
    }
    d.execution_device = "CPU";
    d.selected_predicted_cost_ms = best_cpu;
    d.routing_reason = std::string(gpu_usable ? "B200_CALIBRATED_CPU_SELECTED: " : "B200_CALIBRATED_GPU_UNAVAILABLE: ") +
                       costs;
    return d;
}

}  // namespace bharatopt
