// Drop-in parity tests, written for the reference's own test harness
// (tests/test_harness.hpp of the reference) and linked into dropin_tests.
//
// The reference's tests run GPUFirstOrderSolver on one model only (FO_23); these
// run the same models through both FirstOrderLPSolver backends and require the
// B200 reference engine to return what CPUFirstOrderSolver returns: the same
// status, the same iteration count, and bit-identical primal and dual vectors
// and objective.  They also exercise the Halpern engine through the drop-in and
// the router, judged by the reference's SolutionVerifier.
#include "test_harness.hpp"

#include <bharatopt/benchmark_framework.hpp>
#include <bharatopt/dual_revised_simplex.hpp>
#include <bharatopt/execution_router.hpp>
#include <bharatopt/first_order_solver.hpp>
#include <bharatopt/gpu_backend.hpp>
#include <bharatopt/solution_verifier.hpp>

#include <cmath>
#include <string>

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
    // dual simplex gives the objective it must match, the verifier judges the point
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
