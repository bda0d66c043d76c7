// B200-calibrated cost model and adaptive routing for the reference's execution
// router, supplied through the reference's own extension points:
//
//   B200CostEstimator   implements bharatopt::ICostEstimator
//                       (include/bharatopt/cost_estimator.hpp:126-131).  It replaces
//                       the laptop-calibrated first-order formulas of
//                       AnalyticalCostEstimator::estimate (src/cost_estimator.cpp:175-209)
//                       with costs measured on one B200 and on the reference's own CPU
//                       PDHG; the simplex estimates are the reference's, unchanged.
//   B200ExecutionRouter derives from bharatopt::ExecutionRouter
//                       (include/bharatopt/execution_router.hpp:97-115) and replaces the
//                       fixed size threshold of the adaptive rule
//                       (src/execution_router.cpp:128-139: n >= 1000 or nnz >= 10000 or a
//                       CPU cost above 5 s) by a comparison of the calibrated estimates:
//                       GPU PDHG when the device is usable and its predicted time is the
//                       smallest.  Forced modes and the MILP branch keep the reference's
//                       behaviour; solve() is the reference's (it calls decide()).
//
// A caller opts in by constructing the router with these classes, e.g.
//   bharatopt::B200ExecutionRouter router(cfg);
#pragma once

#include <memory>
#include <vector>

#include <bharatopt/cost_estimator.hpp>
#include <bharatopt/execution_router.hpp>

namespace bharatopt {

// Measured constants of the cost model (one B200, clocks 1965 MHz; the host side on the
// GPU box's CPU).  Times in milliseconds.
struct B200Calibration {
    // host prologue the drop-in runs before the engine (the reference's validator and
    // presolve, src/first_order_solver.cpp:19-34): 90 + 174 ms at 800k nonzeros
    double host_prologue_ms_per_nnz = 3.3e-4;
    // upload + first-solve set-up on the device (transpose, renumbering, Ruiz scaling, SELL
    // copies, tuner): about 240 ms at 8.2M nonzeros on the block-angular LP
    double gpu_setup_ms = 20.0;
    double gpu_setup_ms_per_nnz = 2.7e-5;
    // one Halpern PDHG iteration: a floor of two graph-replayed kernels on a small LP,
    // plus 61 us per 8.0M nonzeros (FP32 SELL kernels on the block-angular LP)
    double gpu_iter_ms = 0.005;
    double gpu_iter_ms_per_nnz = 7.6e-9;
    // iterations to 1e-6 relative KKT on the measured families (random sparse 5,056,
    // block-angular 6,784): the model's typical count
    double gpu_iterations = 8000.0;
    // the reference's CPU PDHG: 2.95 ms per iteration at 800k nonzeros, one core; it runs to
    // its own max_iterations (50,000 by default) on these LPs
    double cpu_pdhg_iter_ms_per_nnz = 3.7e-6;
    double cpu_pdhg_iter_ms = 0.002;
    double cpu_pdhg_iterations = 50000.0;
};

class B200CostEstimator : public ICostEstimator {
public:
    explicit B200CostEstimator(B200Calibration cal = {}) : cal_(cal) {}
    CostEstimate estimate(const WorkloadFeatures& features, BenchmarkSolverType solver) const override;
    std::vector<CostEstimate> estimate_all(const WorkloadFeatures& features) const override;
    const B200Calibration& calibration() const { return cal_; }

private:
    B200Calibration cal_;
    AnalyticalCostEstimator simplex_;  // the reference's own simplex cost model
};

class B200ExecutionRouter : public ExecutionRouter {
public:
    explicit B200ExecutionRouter(RoutingConfiguration config = {}, std::shared_ptr<ICostEstimator> estimator = nullptr);
    RoutingDecision decide(const LPModel& model, const WorkloadFeatures& features,
                           const std::vector<CostEstimate>& estimates) override;
};

}  // namespace bharatopt
