// Batched branch-and-bound over the B200 PDHG engine (see b200_branch_and_bound.hpp).
#include "b200_branch_and_bound.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include <bharatopt/milp_foundation.hpp>
#include <bharatopt/revised_simplex.hpp>
#include <bharatopt/sparse_matrix.hpp>

#include "../../include/b2p.h"

namespace bharatopt {

namespace {

// min c.x  s.t.  A x (<= | =) b,  lb <= x <= ub  of the relaxation, variables in model order
struct StdForm {
    int m = 0, n = 0;
    std::vector<int32_t> rowptr, colidx;
    std::vector<double> vals, b, c, lb, ub;
    std::vector<uint8_t> is_eq;
    std::vector<uint8_t> integral;  // 1 for INTEGER / BINARY variables
};

bool build_std(const LPModel& model, StdForm& s, std::string& why) {
    LPRelaxation rel = MilpFoundation::extract_relaxation(model);
    const LPModel& r = rel.relaxation_model;
    s.m = (int)r.num_constraints();
    s.n = (int)r.num_variables();
    if (s.m == 0 || s.n == 0) {
        why = "the relaxation has no rows or no columns";
        return false;
    }
    const double mult = model.sense() == ObjectiveSense::MINIMIZE ? 1.0 : -1.0;
    s.c.resize(s.n);
    s.lb.resize(s.n);
    s.ub.resize(s.n);
    s.integral.assign(s.n, 0);
    for (int j = 0; j < s.n; ++j) {
        const Variable& v = r.get_variable(j);
        s.c[j] = mult * v.obj_coeff;
        s.lb[j] = v.lower_bound;
        s.ub[j] = v.upper_bound;
        const VariableType t = model.get_variable(rel.mapping.lp_to_milp[j]).type;
        s.integral[j] = (t == VariableType::INTEGER || t == VariableType::BINARY) ? 1 : 0;
    }
    COOMatrix coo(s.m, s.n);
    s.b.resize(s.m);
    s.is_eq.assign(s.m, 0);
    for (int i = 0; i < s.m; ++i) {
        const Constraint& con = r.get_constraint(i);
        double sign = 1.0;
        if (con.sense == ConstraintSense::RANGED) {
            why = "ranged rows are not supported";
            return false;
        }
        if (con.sense == ConstraintSense::GREATER_EQUAL) sign = -1.0;
        if (con.sense == ConstraintSense::EQUAL) s.is_eq[i] = 1;
        s.b[i] = sign * con.rhs;
        for (const auto& t : con.terms) coo.add_entry(i, t.first, sign * t.second);
    }
    CSRMatrix A = CSRMatrix::from_coo(coo);
    s.rowptr.assign(A.row_offsets().begin(), A.row_offsets().end());
    s.colidx.assign(A.col_indices().begin(), A.col_indices().end());
    s.vals.assign(A.values().begin(), A.values().end());
    return true;
}

struct Node {
    std::vector<double> lb, ub;  // bounds of this node
    std::vector<double> x, y;    // parent's relaxation answer (warm start); empty at the root
    double bound = -INFINITY;    // lower bound of the relaxation (min form)
    int depth = 0;
    long long id = 0;
};

struct BoundOrder {  // best bound first
    bool operator()(const Node& a, const Node& b) const { return a.bound > b.bound; }
};

struct Solved {
    int status = B2P_STATUS_NUMERICAL_FAILURE;
    double pobj = 0, obj_err = 0;
    std::vector<double> x, y;
};

// One batched solve of the relaxations with the given bounds (warm starts optional).
int solve_batch(void* ctx, const StdForm& s, const std::vector<const Node*>& nodes, const B200BnBOptions& o,
                std::vector<Solved>& out) {
    const int cnt = (int)nodes.size();
    const size_t N = (size_t)s.n, M = (size_t)s.m;
    std::vector<double> b(M * cnt), c(N * cnt), lb(N * cnt), ub(N * cnt), x0(N * cnt), y0(M * cnt);
    std::vector<uint8_t> eq(M * cnt);
    std::vector<int32_t> inst(cnt, 0);
    bool warm = true;
    for (int k = 0; k < cnt; ++k) {
        std::copy(s.b.begin(), s.b.end(), b.begin() + k * M);
        std::copy(s.c.begin(), s.c.end(), c.begin() + k * N);
        std::copy(s.is_eq.begin(), s.is_eq.end(), eq.begin() + k * M);
        std::copy(nodes[k]->lb.begin(), nodes[k]->lb.end(), lb.begin() + k * N);
        std::copy(nodes[k]->ub.begin(), nodes[k]->ub.end(), ub.begin() + k * N);
        if (nodes[k]->x.size() == N && nodes[k]->y.size() == M) {
            std::copy(nodes[k]->x.begin(), nodes[k]->x.end(), x0.begin() + k * N);
            std::copy(nodes[k]->y.begin(), nodes[k]->y.end(), y0.begin() + k * M);
        } else {
            warm = false;
        }
    }
    const int32_t mm = s.m, nn = s.n;
    const int64_t off[2] = {0, (int64_t)s.vals.size()};
    int st = b2p_batch_upload(ctx, 1, &mm, &nn, off, s.rowptr.data(), s.colidx.data(), s.vals.data(), cnt, inst.data(),
                              b.data(), c.data(), lb.data(), ub.data(), eq.data());
    if (st != B2P_OK) return st;
    b2p_params p;
    b2p_params_default(&p);
    p.engine = B2P_ENGINE_HALPERN;
    p.precision = o.precision;
    p.eps_rel_kkt = o.eps_rel_kkt;
    p.eps_objective = o.eps_objective;
    p.max_iterations = o.max_iterations;
    std::vector<int32_t> status(cnt);
    std::vector<double> x(N * cnt), y(M * cnt), pobj(cnt), err(cnt);
    b2p_result sum;
    st = b2p_batch_solve(ctx, &p, warm ? x0.data() : nullptr, warm ? y0.data() : nullptr, nullptr, status.data(),
                         nullptr, nullptr, nullptr, x.data(), y.data(), &sum);
    if (st != B2P_OK) return st;
    st = b2p_batch_objectives(ctx, pobj.data(), nullptr, err.data());
    if (st != B2P_OK) return st;
    out.assign(cnt, Solved());
    for (int k = 0; k < cnt; ++k) {
        out[k].status = status[k];
        out[k].pobj = pobj[k];
        out[k].obj_err = err[k];
        out[k].x.assign(x.begin() + k * N, x.begin() + (k + 1) * N);
        out[k].y.assign(y.begin() + k * M, y.begin() + (k + 1) * M);
    }
    return B2P_OK;
}

// most fractional integer variable of x within the node's bounds (-1: none above tolerance)
int branching_variable(const StdForm& s, const std::vector<double>& x, double tol, double* val) {
    int best = -1;
    double best_frac = tol;
    for (int j = 0; j < s.n; ++j) {
        if (!s.integral[j]) continue;
        const double f = std::fabs(x[j] - std::round(x[j]));
        if (f > best_frac) {
            best_frac = f;
            best = j;
            *val = x[j];
        }
    }
    return best;
}

}  // namespace

BnBResult B200BranchAndBound::solve(const LPModel& model) {
    const auto t0 = std::chrono::high_resolution_clock::now();
    auto elapsed_ms = [&]() {
        return std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
    };
    BnBResult res;
    res.telemetry.warm_start_mode = config_.warm_start_mode;
    batches_ = 0;
    auto finish = [&](BnBSolverStatus st, const std::string& msg) {
        res.status = st;
        res.status_message = msg;
        res.telemetry.status = st;
        res.telemetry.total_solve_time_ms = elapsed_ms();
        return res;
    };
    StdForm s;
    std::string why;
    if (!build_std(model, s, why)) return finish(BnBSolverStatus::UNSUPPORTED_MODEL, "B200 batched B&B: " + why);
    void* ctx = nullptr;
    if (b2p_ctx_create(0, &ctx) != B2P_OK || !ctx)
        return finish(BnBSolverStatus::UNSUPPORTED_MODEL, "B200 batched B&B: no usable GPU");
    struct CtxGuard {
        void* c;
        ~CtxGuard() { b2p_ctx_destroy(c); }
    } guard{ctx};
    const double mult = model.sense() == ObjectiveSense::MINIMIZE ? 1.0 : -1.0;
    RevisedSimplex objective;  // the reference's objective of an original-space point
    const double tol_int = config_.integrality_tolerance;
    double incumbent = INFINITY;  // min form
    std::vector<double> best_x;
    size_t unresolved = 0;

    // root
    Node root;
    root.lb = s.lb;
    root.ub = s.ub;
    std::vector<Solved> out;
    int st = solve_batch(ctx, s, {&root}, options_, out);
    batches_++;
    res.telemetry.root_relaxation_time_ms = elapsed_ms();
    res.telemetry.nodes_created = 1;
    if (st != B2P_OK)
        return finish(BnBSolverStatus::NUMERICAL_FAILURE, std::string("B200 batched B&B: ") + b2p_last_error(ctx));
    if (out[0].status == B2P_STATUS_INFEASIBLE_DETECTED)
        return finish(BnBSolverStatus::INFEASIBLE, "Root LP relaxation is infeasible (dual ray); MILP is infeasible.");
    if (out[0].status == B2P_STATUS_UNBOUNDED_DETECTED)
        return finish(BnBSolverStatus::UNRESOLVED, "Root LP relaxation is unbounded (primal ray).");
    if (out[0].status != B2P_STATUS_OPTIMAL)
        return finish(BnBSolverStatus::NUMERICAL_FAILURE, "Root LP relaxation did not converge.");

    std::priority_queue<Node, std::vector<Node>, BoundOrder> open;
    long long next_id = 1;
    // a solved node: pruned (infeasible, by bound, or unresolved), a new incumbent, or open
    auto absorb = [&](Node& nd, Solved& sv) {
        if (sv.status == B2P_STATUS_INFEASIBLE_DETECTED) {
            res.telemetry.nodes_pruned_infeasibility++;
            return;
        }
        if (sv.status != B2P_STATUS_OPTIMAL) {
            unresolved++;
            return;
        }
        // a lower bound on this node's optimum despite the approximate answer
        nd.bound = sv.pobj - sv.obj_err * std::max(1.0, std::fabs(sv.pobj));
        if (nd.bound >= incumbent - config_.objective_tolerance * std::max(1.0, std::fabs(incumbent))) {
            res.telemetry.nodes_pruned_bound++;
            return;
        }
        double v = 0.0;
        const int j = branching_variable(s, sv.x, tol_int, &v);
        if (j < 0) {  // integral within tolerance: round the integer variables and verify
            std::vector<double> xr = sv.x;
            for (int q = 0; q < s.n; ++q)
                if (s.integral[q]) xr[q] = std::round(xr[q]);
            IntegerVerificationResult ver = MilpFoundation::verify_integer_feasibility(model, xr, tol_int);
            res.telemetry.integer_feasible_nodes++;
            if (!ver.is_integer_feasible) {
                unresolved++;
                return;
            }
            const double z = mult * objective.recompute_original_objective(model, xr);
            if (z < incumbent) {
                incumbent = z;
                best_x = xr;
                res.incumbent.has_incumbent = true;
                res.incumbent.objective_value = mult * z;
                res.incumbent.solution = xr;
                res.incumbent.originating_node_id = nd.id;
                res.incumbent.verification = ver;
                res.telemetry.incumbent_updates++;
            }
            return;
        }
        res.telemetry.fractional_nodes++;
        nd.x = std::move(sv.x);
        nd.y = std::move(sv.y);
        open.push(std::move(nd));
    };
    absorb(root, out[0]);
    res.telemetry.nodes_processed = 1;

    while (!open.empty()) {
        if (res.telemetry.nodes_processed >= config_.max_nodes || elapsed_ms() > config_.time_limit_ms)
            return finish(BnBSolverStatus::LIMIT_REACHED, "B200 batched B&B: node or time limit reached.");
        // up to batch_nodes open nodes, best bound first; their children form one batch
        std::vector<Node> kids;
        for (int k = 0; k < options_.batch_nodes && !open.empty(); ++k) {
            Node nd = open.top();
            open.pop();
            if (nd.bound >= incumbent - config_.objective_tolerance * std::max(1.0, std::fabs(incumbent))) {
                res.telemetry.nodes_pruned_bound++;
                continue;
            }
            double v = 0.0;
            const int j = branching_variable(s, nd.x, tol_int, &v);
            if (j < 0) continue;  // cannot happen: integral nodes never enter the queue
            for (int side = 0; side < 2; ++side) {
                Node ch;
                ch.lb = nd.lb;
                ch.ub = nd.ub;
                if (side == 0) ch.ub[j] = std::min(ch.ub[j], std::floor(v));
                else ch.lb[j] = std::max(ch.lb[j], std::ceil(v));
                if (ch.lb[j] > ch.ub[j] + 1e-9) {  // contradictory bounds
                    res.telemetry.nodes_pruned_infeasibility++;
                    continue;
                }
                ch.x = nd.x;
                ch.y = nd.y;
                ch.depth = nd.depth + 1;
                ch.id = next_id++;
                res.telemetry.max_tree_depth = std::max(res.telemetry.max_tree_depth, ch.depth);
                kids.push_back(std::move(ch));
            }
        }
        if (kids.empty()) continue;
        std::vector<const Node*> ptrs;
        for (auto& k : kids) ptrs.push_back(&k);
        res.telemetry.nodes_created += kids.size();
        res.telemetry.warm_starts_attempted += kids.size();
        st = solve_batch(ctx, s, ptrs, options_, out);
        batches_++;
        if (st != B2P_OK)
            return finish(BnBSolverStatus::NUMERICAL_FAILURE, std::string("B200 batched B&B: ") + b2p_last_error(ctx));
        res.telemetry.warm_starts_accepted += kids.size();
        for (size_t k = 0; k < kids.size(); ++k) {
            res.telemetry.nodes_processed++;
            absorb(kids[k], out[k]);
        }
    }
    res.telemetry.final_incumbent_obj = res.incumbent.objective_value;
    res.telemetry.best_open_bound = res.incumbent.objective_value;
    if (!res.incumbent.has_incumbent)
        return finish(unresolved ? BnBSolverStatus::LIMIT_REACHED : BnBSolverStatus::INFEASIBLE,
                      unresolved ? "B200 batched B&B: no incumbent; some relaxations did not converge."
                                 : "Every node is infeasible or pruned; MILP is infeasible.");
    res.objective_value = res.incumbent.objective_value;
    res.solution = best_x;
    if (unresolved)
        return finish(BnBSolverStatus::LIMIT_REACHED,
                      "B200 batched B&B: incumbent found; " + std::to_string(unresolved) +
                          " node relaxations did not converge and were dropped.");
    return finish(BnBSolverStatus::OPTIMAL, "B200 batched B&B: optimal (" + std::to_string(batches_) +
                                                " batched relaxation solves).");
}

}  // namespace bharatopt
