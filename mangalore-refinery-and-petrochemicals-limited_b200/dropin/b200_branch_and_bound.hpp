// Branch-and-bound whose node LP relaxations are solved in batches on the B200.
//
// The reference's BranchAndBoundEngine (include/bharatopt/branch_and_bound.hpp:138-170,
// src/branch_and_bound.cpp) solves one node relaxation at a time with the dual simplex,
// warm-started from the parent's basis (LPWarmStartState, branch_and_bound.hpp:50-58).
// This engine keeps the reference's configuration, result and telemetry types and its
// branching rule (most fractional variable, children x_j <= floor and x_j >= ceil), but
// processes the open nodes a frontier at a time: each round takes up to `batch_nodes`
// open nodes in best-bound order, creates their children, and solves all child
// relaxations in one batched PDHG launch (b2p_batch_solve) that shares the constraint
// matrix and gives every child its own bounds, warm-started from its parent's primal and
// dual answer (the first-order counterpart of the parent basis).  Infeasible children are
// pruned on the engine's dual-ray certificate; a child's bound for pruning is its primal
// objective minus the device's FP64 bound on the objective error, so approximate
// relaxation answers never prune a node that could hold a better solution.
#pragma once

#include <cstdint>

#include <bharatopt/branch_and_bound.hpp>
#include <bharatopt/lp_model.hpp>

namespace bharatopt {

struct B200BnBOptions {
    int batch_nodes = 64;           // open nodes expanded per round (up to 2x children per batch)
    double eps_rel_kkt = 1e-8;      // node relaxations: relative KKT tolerance
    double eps_objective = 1e-8;    // and the objective-accuracy stop
    int64_t max_iterations = 400000;
    int precision = 0;              // B2P_FP64
};

class B200BranchAndBound {
public:
    explicit B200BranchAndBound(BnBConfig config = BnBConfig(), B200BnBOptions options = {})
        : config_(config), options_(options) {}
    // Same contract as BranchAndBoundEngine::solve: OPTIMAL with the incumbent, INFEASIBLE,
    // LIMIT_REACHED (node or time limit, or nodes whose relaxation did not converge were
    // dropped), UNRESOLVED (unbounded root relaxation), NUMERICAL_FAILURE,
    // UNSUPPORTED_MODEL (ranged rows, no rows, or no usable GPU).
    BnBResult solve(const LPModel& model);
    size_t batches_solved() const { return batches_; }

private:
    BnBConfig config_;
    B200BnBOptions options_;
    size_t batches_ = 0;
};

}  // namespace bharatopt
