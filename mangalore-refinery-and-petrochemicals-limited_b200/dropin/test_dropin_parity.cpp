// Drop-in parity tests, written for the reference's own test harness
// (tests/test_harness.hpp of the reference) and linked into dropin_tests.
//
// The reference's tests run GPUFirstOrderSolver on one model only (FO_23); these
// run the same models through both FirstOrderLPSolver backends and require the
// B200 reference engine to return what CPUFirstOrderSolver returns: the same
// status, the same iteration count, and bit-identical primal and dual vectors
// and objective.  They also exercise the Halpern engine through the drop-in and
// the router, checked by the reference's SolutionVerifier.
#include "test_harness.hpp"

#include <bharatopt/benchmark_framework.hpp>
#include <bharatopt/branch_and_bound.hpp>
#include <bharatopt/milp_foundation.hpp>
#include <bharatopt/dual_revised_simplex.hpp>
#include <bharatopt/execution_router.hpp>
#include <bharatopt/first_order_solver.hpp>
#include <bharatopt/gpu_backend.hpp>
#include <bharatopt/solution_verifier.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <string>

#include "b200_branch_and_bound.hpp"
#include "b200_router.hpp"
#include "b2p_dropin.hpp"

using namespace bharatopt;

namespace {

FirstOrderSolverResult run(const LPModel& m, FirstOrderBackendType backend, size_t max_iterations = 50000) {
    FirstOrderSolverOptions o;
    o.backend_type = backend;
    o.max_iterations = max_iterations;
    FirstOrderLPSolver solver(o);
    return solver.solve(m);
}

bool same_bits(const std::vector<real_t>& a, const std::vector<real_t>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (!(a[i] == b[i] || (std::isnan(a[i]) && std::isnan(b[i])))) return false;
    return true;
}

LPModel generated(const std::string& shape, size_t n, size_t m, uint64_t seed, double density = 0.05) {
    BenchmarkInstanceConfig cfg;
    cfg.instance_id = "dropin_" + shape + "_" + std::to_string(seed);
    cfg.num_variables = n;
    cfg.num_constraints = m;
    cfg.seed = seed;
    cfg.shape_type = shape;
    cfg.target_density = density;
    return BenchmarkGenerator::generate_instance(cfg);
}

}  // namespace

TEST_CASE(DropIn_01_BackendIsARealB200) {
    GpuBackend& gpu = GpuBackend::instance();
    EXPECT_EQ(gpu.initialize(), GPUStatus::SUCCESS);
    EXPECT_TRUE(gpu.is_available());
    EXPECT_EQ(gpu.device_info().compute_capability_major, 10);
    EXPECT_TRUE(gpu.device_info().device_name.find("B200") != std::string::npos);
}

TEST_CASE(DropIn_02_GeneratedModelsBitIdentical) {
    const char* shapes[] = {"square", "banded", "block_sparse", "diagonal"};
    uint64_t seed = 7;
    for (const char* shape : shapes) {
        for (size_t k = 0; k < 2; ++k, ++seed) {
            LPModel model = generated(shape, 60 + 40 * k, 30 + 20 * k, seed, 0.08);
            for (size_t max_it : {size_t(137), size_t(50000)}) {
                FirstOrderSolverResult c = run(model, FirstOrderBackendType::CPU_FIRST_ORDER, max_it);
                FirstOrderSolverResult g = run(model, FirstOrderBackendType::GPU_FIRST_ORDER, max_it);
                EXPECT_EQ(c.status, g.status);
                EXPECT_EQ(c.stats.iterations, g.stats.iterations);
                EXPECT_TRUE(same_bits(c.primal_solution, g.primal_solution));
                EXPECT_TRUE(same_bits(c.dual_solution, g.dual_solution));
                EXPECT_TRUE(c.objective_value == g.objective_value);
                EXPECT_TRUE(c.stats.constraint_violation == g.stats.constraint_violation);
            }
        }
    }
}

TEST_CASE(DropIn_03_HandLPOnGpu) {
    // tests/test_first_order_solver.cpp:268-286 of the reference, on the GPU backend
    LPModel model("hand_lp_gpu");
    model.set_sense(ObjectiveSense::MAXIMIZE);
    index_t x = model.add_variable("x", 0.0, BHARATOPT_INFINITY, 3.0);
    index_t y = model.add_variable("y", 0.0, BHARATOPT_INFINITY, 5.0);
    model.add_constraint("c1", {{x, 2.0}, {y, 1.0}}, ConstraintSense::LESS_EQUAL, 8.0);
    model.add_constraint("c2", {{x, 1.0}, {y, 2.0}}, ConstraintSense::LESS_EQUAL, 8.0);
    FirstOrderSolverResult g = run(model, FirstOrderBackendType::GPU_FIRST_ORDER);
    FirstOrderSolverResult c = run(model, FirstOrderBackendType::CPU_FIRST_ORDER);
    EXPECT_EQ(g.status, FirstOrderSolverStatus::OPTIMAL);
    EXPECT_NEAR(g.primal_solution[x], 8.0 / 3.0, 1e-2);
    EXPECT_NEAR(g.objective_value, 64.0 / 3.0, 1e-2);
    EXPECT_EQ(g.stats.iterations, c.stats.iterations);
    EXPECT_TRUE(same_bits(c.primal_solution, g.primal_solution));
}

TEST_CASE(DropIn_04_IterationLimitOnGpu) {
    // tests/test_first_order_solver.cpp:361-375 of the reference, on the GPU backend
    LPModel model("iter_limit_gpu");
    model.set_sense(ObjectiveSense::MAXIMIZE);
    index_t x = model.add_variable("x", 0.0, 100.0, 5.0);
    index_t y = model.add_variable("y", 0.0, 100.0, 6.0);
    model.add_constraint("c1", {{x, 1.0}, {y, 1.0}}, ConstraintSense::LESS_EQUAL, 50.0);
    FirstOrderSolverResult g = run(model, FirstOrderBackendType::GPU_FIRST_ORDER, 5);
    EXPECT_EQ(g.status, FirstOrderSolverStatus::MAX_ITERATIONS);
    EXPECT_EQ(g.stats.iterations, static_cast<size_t>(5));
}

TEST_CASE(DropIn_05_HalpernEngineVerified) {
    // the Halpern engine to 1e-9 relative KKT through the drop-in; the reference's own
    // dual simplex gives the objective it must match, the verifier checks the point
    LPModel model = generated("square", 120, 60, 99, 0.1);
    b2p_params p;
    b2p_params_default(&p);
    p.engine = B2P_ENGINE_HALPERN;
    p.precision = B2P_FP64;
    p.eps_rel_kkt = 1e-9;
    bharatopt_b200_set_engine(&p);
    FirstOrderSolverResult g = run(model, FirstOrderBackendType::GPU_FIRST_ORDER, 400000);
    bharatopt_b200_set_engine(nullptr);
    EXPECT_EQ(g.status, FirstOrderSolverStatus::OPTIMAL);
    DualRevisedSimplex simplex;
    DualRevisedSimplexResult s = simplex.solve(model);
    if (s.status == DualRevisedSimplexStatus::OPTIMAL) {
        EXPECT_NEAR(g.objective_value, s.objective_value, 1e-6 * std::max(1.0, std::abs(s.objective_value)));
    }
    VerificationOptions vo;
    vo.feasibility_tolerance = 1e-6;
    SolutionVerifier verifier;
    VerificationResult v = verifier.verify(model, g.primal_solution, g.objective_value, vo);
    EXPECT_TRUE(v.verified);
}

TEST_CASE(DropIn_06_RouterForcedGpuHalpern) {
    LPModel model = generated("block_sparse", 200, 100, 5, 0.05);
    b2p_params p;
    b2p_params_default(&p);
    p.engine = B2P_ENGINE_HALPERN;
    p.precision = B2P_FP64;
    p.eps_rel_kkt = 1e-10;
    bharatopt_b200_set_engine(&p);
    RoutingConfiguration cfg;
    cfg.routing_mode = RoutingMode::FORCE_GPU_FIRST_ORDER;
    cfg.fallback_enabled = false;
    ExecutionRouter router(cfg);
    RoutedSolveResult r = router.solve(model);
    bharatopt_b200_set_engine(nullptr);
    EXPECT_EQ(r.decision.execution_device, "GPU");
    EXPECT_EQ(r.status, "OPTIMAL");
    EXPECT_FALSE(r.fallback_occurred);
    EXPECT_TRUE(r.verification_passed);
}

TEST_CASE(DropIn_07_AdaptiveRouterPicksGpuAtScale) {
    // with a real GPU the adaptive rule (src/execution_router.cpp:130-139) selects GPU PDHG
    LPModel model = generated("square", 1200, 600, 3, 0.01);
    ExecutionRouter router;
    WorkloadFeatures f = router.analyse(model);
    EXPECT_TRUE(f.gpu_available);
    std::vector<CostEstimate> est = router.estimate(f);
    RoutingDecision d = router.decide(model, f, est);
    EXPECT_EQ(d.execution_device, "GPU");
    EXPECT_EQ(d.solver_variant, "GPU_PDHG");
}

namespace {

// A two-variable hand LP of the size of the reference's FO_* models.
LPModel toy_model() {
    LPModel model("toy_router");
    model.set_sense(ObjectiveSense::MAXIMIZE);
    index_t x = model.add_variable("x", 0.0, 10.0, 3.0);
    index_t y = model.add_variable("y", 0.0, 10.0, 5.0);
    model.add_constraint("c1", {{x, 1.0}, {y, 2.0}}, ConstraintSense::LESS_EQUAL, 8.0);
    model.add_constraint("c2", {{x, 3.0}, {y, 1.0}}, ConstraintSense::LESS_EQUAL, 9.0);
    return model;
}

// Features of the block-angular multi-period LP (204k rows, 1M columns, 8.2M nonzeros)
// on top of the features of a small model.
WorkloadFeatures block_angular_scale(WorkloadFeatures f) {
    f.m = f.orig_m = f.reduced_m = 204000;
    f.n = f.orig_n = f.reduced_n = 1000000;
    f.nnz = f.orig_nnz = f.reduced_nnz = 8200000;
    f.density = 8.2e6 / (2.04e5 * 1.0e6);
    f.avg_nnz_per_row = 8.2e6 / 2.04e5;
    f.avg_nnz_per_col = 8.2;
    return f;
}

}  // namespace

TEST_CASE(DropIn_08_CalibratedRouterKeepsToyModelsOnCpu) {
    // the B200-calibrated estimates (not a size threshold) keep an FO-sized model on the CPU
    B200ExecutionRouter router;
    LPModel toy = toy_model();
    WorkloadFeatures f = router.analyse(toy);
    EXPECT_TRUE(f.gpu_available);
    std::vector<CostEstimate> est = router.estimate(f);
    RoutingDecision d = router.decide(toy, f, est);
    EXPECT_EQ(d.execution_device, "CPU");
    EXPECT_TRUE(d.routing_reason.rfind("B200_CALIBRATED_CPU_SELECTED", 0) == 0);
    EXPECT_TRUE(d.predicted_gpu_cost_ms > d.predicted_cpu_cost_ms);
    RoutedSolveResult r = router.solve(toy);
    EXPECT_EQ(r.status, "OPTIMAL");
    EXPECT_NEAR(r.objective_value, 3.0 * 2.0 + 5.0 * 3.0, 1e-6);
}

TEST_CASE(DropIn_09_CalibratedRouterPicksGpuAtBlockAngularScale) {
    B200ExecutionRouter router;
    LPModel toy = toy_model();
    WorkloadFeatures big = block_angular_scale(router.analyse(toy));
    std::vector<CostEstimate> est = router.estimate(big);
    RoutingDecision d = router.decide(toy, big, est);
    EXPECT_EQ(d.execution_device, "GPU");
    EXPECT_EQ(d.solver_variant, "GPU_PDHG");
    EXPECT_TRUE(d.routing_reason.rfind("B200_CALIBRATED_GPU_SELECTED", 0) == 0);
    EXPECT_TRUE(d.predicted_gpu_cost_ms < d.predicted_cpu_cost_ms);
    // the calibrated GPU estimate at this size: seconds, not the laptop formula's minutes
    EXPECT_TRUE(d.predicted_gpu_cost_ms > 1000.0 && d.predicted_gpu_cost_ms < 20000.0);
}

TEST_CASE(RouterB200_01_NoDeviceStaysOnCpu) {
    // without a usable device the calibrated router never selects the GPU path
    B200ExecutionRouter router;
    LPModel toy = toy_model();
    WorkloadFeatures big = block_angular_scale(router.analyse(toy));
    big.gpu_available = false;
    big.cuda_available = false;
    RoutingDecision d = router.decide(toy, big, router.estimate(big));
    EXPECT_EQ(d.execution_device, "CPU");
    EXPECT_TRUE(d.routing_reason.rfind("B200_CALIBRATED_GPU_UNAVAILABLE", 0) == 0);
}

namespace {

// Small MILPs for the batched branch-and-bound, each solved by the reference's
// BranchAndBoundEngine as well.
LPModel milp_three_int() {
    LPModel m("milp_three_int");
    m.set_sense(ObjectiveSense::MAXIMIZE);
    index_t x = m.add_variable("x", 0.0, 10.0, 5.0, VariableType::INTEGER);
    index_t y = m.add_variable("y", 0.0, 10.0, 4.0, VariableType::INTEGER);
    index_t z = m.add_variable("z", 0.0, 10.0, 3.0, VariableType::INTEGER);
    m.add_constraint("r1", {{x, 2.0}, {y, 3.0}, {z, 1.0}}, ConstraintSense::LESS_EQUAL, 5.0);
    m.add_constraint("r2", {{x, 4.0}, {y, 1.0}, {z, 2.0}}, ConstraintSense::LESS_EQUAL, 11.0);
    m.add_constraint("r3", {{x, 3.0}, {y, 4.0}, {z, 2.0}}, ConstraintSense::LESS_EQUAL, 8.0);
    return m;
}

LPModel milp_knapsack(int items, int rows, uint64_t seed) {
    LPModel m("milp_knapsack_" + std::to_string(items));
    m.set_sense(ObjectiveSense::MAXIMIZE);
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        z ^= z << 13;
        z ^= z >> 7;
        z ^= z << 17;
        return (double)(z % 1000) / 1000.0;
    };
    std::vector<index_t> v;
    for (int i = 0; i < items; ++i) v.push_back(m.add_variable("x" + std::to_string(i), 0.0, 1.0, 10.0 + 40.0 * next(),
                                                              VariableType::BINARY));
    for (int r = 0; r < rows; ++r) {
        std::vector<std::pair<index_t, real_t>> t;
        double total = 0.0;
        for (int i = 0; i < items; ++i) {
            const double w = 5.0 + 20.0 * next();
            t.push_back({v[i], w});
            total += w;
        }
        m.add_constraint("cap" + std::to_string(r), t, ConstraintSense::LESS_EQUAL, std::floor(0.4 * total));
    }
    return m;
}

LPModel milp_integer_infeasible() {
    // the relaxation is feasible (x + y = 1.5), no integer point is
    LPModel m("milp_integer_infeasible");
    m.set_sense(ObjectiveSense::MINIMIZE);
    index_t x = m.add_variable("x", 0.0, 5.0, 1.0, VariableType::INTEGER);
    index_t y = m.add_variable("y", 0.0, 5.0, 2.0, VariableType::INTEGER);
    m.add_constraint("half", {{x, 1.0}, {y, 1.0}}, ConstraintSense::EQUAL, 1.5);
    return m;
}

LPModel milp_mixed() {
    // integers and a continuous variable, a >= row and an equality
    LPModel m("milp_mixed");
    m.set_sense(ObjectiveSense::MINIMIZE);
    index_t a = m.add_variable("a", 0.0, 20.0, 3.0, VariableType::INTEGER);
    index_t b = m.add_variable("b", 0.0, 20.0, 2.0, VariableType::INTEGER);
    index_t c = m.add_variable("c", 0.0, 10.0, 1.5, VariableType::CONTINUOUS);
    m.add_constraint("cover", {{a, 2.0}, {b, 1.0}, {c, 1.0}}, ConstraintSense::GREATER_EQUAL, 7.5);
    m.add_constraint("mix", {{a, 1.0}, {b, 3.0}}, ConstraintSense::GREATER_EQUAL, 5.5);
    m.add_constraint("tie", {{a, 1.0}, {b, -1.0}, {c, 1.0}}, ConstraintSense::EQUAL, 0.5);
    return m;
}

void expect_same_milp_answer(const LPModel& model) {
    BranchAndBoundEngine ref;
    BnBResult r = ref.solve(model);
    B200BranchAndBound gpu;
    BnBResult g = gpu.solve(model);
    EXPECT_TRUE(g.status == r.status);
    if (r.status == BnBSolverStatus::OPTIMAL && g.status == BnBSolverStatus::OPTIMAL) {
        EXPECT_NEAR(g.objective_value, r.objective_value, 1e-4 * std::max(1.0, std::fabs(r.objective_value)));
        IntegerVerificationResult v = MilpFoundation::verify_integer_feasibility(model, g.solution, 1e-5);
        EXPECT_TRUE(v.is_integer_feasible);
    }
}

}  // namespace

TEST_CASE(DropIn_10_BatchedBnBMatchesReferenceEngine) {
    expect_same_milp_answer(milp_three_int());
    expect_same_milp_answer(milp_integer_infeasible());
    expect_same_milp_answer(milp_mixed());
    expect_same_milp_answer(milp_knapsack(12, 1, 3));
}

TEST_CASE(DropIn_11_BatchedBnBKnapsackFrontier) {
    // 24 binaries under two capacity rows: many open nodes, solved a frontier per batch
    LPModel model = milp_knapsack(24, 2, 7);
    B200BranchAndBound gpu;
    BnBResult g = gpu.solve(model);
    BranchAndBoundEngine ref;
    BnBResult r = ref.solve(model);
    EXPECT_TRUE(g.status == BnBSolverStatus::OPTIMAL);
    EXPECT_TRUE(r.status == BnBSolverStatus::OPTIMAL);
    EXPECT_NEAR(g.objective_value, r.objective_value, 1e-4 * std::max(1.0, std::fabs(r.objective_value)));
    EXPECT_TRUE(gpu.batches_solved() < g.telemetry.nodes_processed);  // several nodes per launch
}

namespace {

// Random sparse LP in the model API: m rows (<= and >=, and with `ranged` every third row
// ranged), n columns in [0, 10], about k nonzeros per column, feasible at x0 = 1.
LPModel random_model(int m, int n, int k, uint64_t seed, bool ranged) {
    LPModel model("direct_setup_" + std::to_string(m));
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + 7;
    auto u01 = [&]() {
        z ^= z << 13;
        z ^= z >> 7;
        z ^= z << 17;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    std::vector<index_t> v(n);
    for (int j = 0; j < n; ++j) v[j] = model.add_variable("x" + std::to_string(j), 0.0, 10.0, 2.0 * u01() - 1.0);
    std::vector<std::vector<std::pair<index_t, real_t>>> rows(m);
    for (int j = 0; j < n; ++j)
        for (int q = 0; q < k; ++q) {
            auto& r = rows[(size_t)(u01() * m) % m];
            if (r.empty() || r.back().first != v[j]) r.push_back({v[j], 0.5 + u01()});  // no repeated term
        }
    for (int i = 0; i < m; ++i) {
        double act = 0.0;
        for (auto& t : rows[i]) act += t.second;
        if (i % 3 == 0 || (!ranged && i % 3 == 2))
            model.add_constraint("r" + std::to_string(i), rows[i], ConstraintSense::LESS_EQUAL, act + 1.0);
        else if (i % 3 == 1)
            model.add_constraint("r" + std::to_string(i), rows[i], ConstraintSense::GREATER_EQUAL, act - 1.0);
        else {
            index_t c = model.add_constraint("r" + std::to_string(i), ConstraintSense::RANGED, act - 0.5, act + 0.5);
            for (auto& t : rows[i]) model.set_coeff(c, t.first, t.second);
        }
    }
    return model;
}

double ms_since(std::chrono::high_resolution_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t).count();
}

}  // namespace

TEST_CASE(DropIn_12_DirectSetupMatchesAndSkipsHostPresolve) {
    // same LP through the reference front end and through the direct setup, Halpern FP64
    b2p_params p;
    b2p_params_default(&p);
    p.engine = B2P_ENGINE_HALPERN;
    p.precision = B2P_FP64;
    p.eps_rel_kkt = 1e-9;
    p.max_iterations = 400000;
    bharatopt_b200_set_engine(&p);
    LPModel small = random_model(300, 900, 3, 11, false);
    FirstOrderSolverOptions o;
    o.backend_type = FirstOrderBackendType::GPU_FIRST_ORDER;
    o.max_iterations = 400000;
    bharatopt_b200_set_setup(0);
    FirstOrderSolverResult a = FirstOrderLPSolver(o).solve(small);
    bharatopt_b200_set_setup(1);
    FirstOrderSolverResult b = FirstOrderLPSolver(o).solve(small);
    EXPECT_EQ(a.status, FirstOrderSolverStatus::OPTIMAL);
    EXPECT_EQ(b.status, FirstOrderSolverStatus::OPTIMAL);
    EXPECT_NEAR(b.objective_value, a.objective_value, 1e-6 * std::max(1.0, std::fabs(a.objective_value)));
    SolutionVerifier ver;
    VerificationOptions vo;
    vo.feasibility_tolerance = 1e-5;
    EXPECT_TRUE(ver.verify(small, b.primal_solution, vo).verified);
    // ranged rows: the direct setup keeps both ends (the reference front end keeps only the
    // lower end), checked by the reference's verifier, which reads both
    LPModel rng = random_model(300, 900, 3, 13, true);
    FirstOrderSolverResult e = FirstOrderLPSolver(o).solve(rng);
    EXPECT_EQ(e.status, FirstOrderSolverStatus::OPTIMAL);
    vo.check_objective = false;
    EXPECT_TRUE(ver.verify(rng, e.primal_solution, vo).verified);
    // setup time at 800k nonzeros: a few iterations so the host front end dominates
    LPModel big = random_model(20000, 100000, 8, 12, false);
    p.max_iterations = 64;
    p.eps_rel_kkt = 0.0;
    bharatopt_b200_set_engine(&p);
    o.max_iterations = 64;
    bharatopt_b200_set_setup(0);
    auto t0 = std::chrono::high_resolution_clock::now();
    FirstOrderSolverResult c = FirstOrderLPSolver(o).solve(big);
    const double ref_ms = ms_since(t0);
    bharatopt_b200_set_setup(1);
    t0 = std::chrono::high_resolution_clock::now();
    FirstOrderSolverResult d = FirstOrderLPSolver(o).solve(big);
    const double direct_ms = ms_since(t0);
    bharatopt_b200_set_setup(-1);
    bharatopt_b200_set_engine(nullptr);
    std::printf("  [direct setup] 20000 x 100000, 800k nnz: reference front end + 64 iterations %.1f ms, "
                "direct setup + 64 iterations %.1f ms\n", ref_ms, direct_ms);
    EXPECT_EQ(c.status, FirstOrderSolverStatus::MAX_ITERATIONS);
    EXPECT_EQ(d.status, FirstOrderSolverStatus::MAX_ITERATIONS);
    EXPECT_TRUE(direct_ms * 2.0 < ref_ms);
}
