"""Reference engine on the GPU: iterate-for-iterate the reference PDHG.

Parity bar: bit-identical x, y, status, iteration count and violations against
the compiled reference's golden traces and against the oracle restatement."""
from __future__ import annotations

import numpy as np
import pytest

import fo_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["rs_c0", "rs_small", "rs_ge"])
@pytest.mark.parametrize("k", [1, 7, 100, 1000])
def test_reference_engine_matches_reference_traces(ctx, golden, golden_std, name, k):
    lp = golden_std(name)
    ctx.upload(lp)
    res, x, y = ctx.solve(engine="reference", max_iterations=k)
    meta = golden["meta"][f"{name}/K{k}"]
    assert res["status"] == meta["status"]
    assert res["iterations"] == meta["iterations"]
    assert np.array_equal(y, golden["arrays"][f"{name}/K{k}/y"])
    assert np.array_equal(x, golden["arrays"][f"{name}/K{k}/x"])
    assert res["constraint_violation"] == meta["constraint_violation"]
    assert res["bound_violation"] == meta["bound_violation"]


@pytest.mark.parametrize("case", fo_cases.CASES, ids=[c[0] for c in fo_cases.CASES])
def test_reference_engine_known_answers(ctx, golden, golden_std, case):
    name, _, lp, exp = case
    meta = golden["meta"][name]
    if meta["sf_status"] != 0:
        pytest.skip("reference solves this case in presolve; covered by the drop-in tests")
    ctx.upload(golden_std(name))
    res, x, y = ctx.solve(engine="reference", max_iterations=meta["max_iterations"])
    assert res["status"] == meta["status"] and res["iterations"] == meta["iterations"]
    assert np.array_equal(y, golden["arrays"][f"{name}/y"])


def test_reference_engine_full_run_matches_oracle(ctx, oracle, golden_std):
    """The whole default 50000-iteration run of the 300 x 1000 LP, bit for bit."""
    lp = golden_std("rs_c0")
    ctx.upload(lp)
    res, x, y = ctx.solve(engine="reference")
    o = oracle.ref_pdhg(lp)
    assert res["status"] == o["status"] == "MAX_ITERATIONS"
    assert res["iterations"] == o["iterations"] == 50000
    assert np.array_equal(x, o["x_final"]) and np.array_equal(y, o["y_last"])
    assert res["used_average"] == o["used_average"]


@pytest.mark.parametrize("opts", [dict(check_frequency=7, max_iterations=1000),
                                  dict(adaptive_step_size=0, primal_step_size=0.003, dual_step_size=0.002,
                                       max_iterations=777),
                                  dict(max_iterations=0), dict(max_iterations=250, check_frequency=1000)])
def test_reference_engine_options(ctx, oracle, lpgen, opts):
    lp = lpgen.random_sparse(m=60, n=150, nnz_per_col=3, seed=21).standard()
    ctx.upload(lp)
    res, x, y = ctx.solve(engine="reference", **opts)
    o = oracle.ref_pdhg(lp, max_iterations=opts.get("max_iterations", 50000),
                        check_frequency=opts.get("check_frequency", 100),
                        adaptive=bool(opts.get("adaptive_step_size", 1)),
                        primal_step=opts.get("primal_step_size", 0.01), dual_step=opts.get("dual_step_size", 0.01))
    assert res["status"] == o["status"] and res["iterations"] == o["iterations"]
    assert np.array_equal(x, o["x_final"]) and np.array_equal(y, o["y_last"])


@pytest.mark.parametrize("step,want", [(1.0, "NUMERICAL_FAILURE"), (50.0, "OPTIMAL")])
def test_reference_engine_divergence_semantics(ctx, oracle, lpgen, step, want):
    """Free variables and fixed large steps: the iterates overflow.  At step 1 the row violation
    exceeds 1e15 -> NUMERICAL_FAILURE (first_order_solver.cpp:232-236).  At step 50 they become NaN,
    which std::max drops, so the reference reports OPTIMAL; the GPU engine reproduces both."""
    lp = lpgen.random_sparse(m=30, n=90, nnz_per_col=3, seed=4).standard()
    lp.lb[:] = -np.inf
    lp.ub[:] = np.inf
    ctx.upload(lp)
    res, _, _ = ctx.solve(engine="reference", adaptive_step_size=0, primal_step_size=step, dual_step_size=step,
                          max_iterations=5000)
    o = oracle.ref_pdhg(lp, max_iterations=5000, adaptive=False, primal_step=step, dual_step=step)
    assert o["status"] == want
    assert res["status"] == o["status"] and res["iterations"] == o["iterations"]
