"""Pins the oracle before anything is checked against it (CPU only).

* pdhg_oracle.c (the C restatement of CPUFirstOrderSolver::solve) must
  reproduce the compiled reference bit for bit: the committed golden traces
  (generated from the reference by tests/golden/make_golden.py) and, when
  oracle/_ref is built here, fresh seeds run through the live reference.
* The oracle SpMV / transpose-SpMV equal CSRMatrix::multiply / multiply_transpose.
* The FP64 KKT checker gives ~0 at the HiGHS optimum and the restated
  engine algorithm (pdlp_oracle.halpern_pdhg) reaches the HiGHS objective.
"""
from __future__ import annotations

import numpy as np
import pytest

import fo_cases

SEEDED = ["rs_c0", "rs_small", "rs_ge"]


@pytest.mark.parametrize("name", SEEDED)
@pytest.mark.parametrize("k", [1, 7, 100, 1000])
def test_oracle_matches_reference_traces(oracle, golden, golden_std, name, k):
    lp = golden_std(name)
    meta = golden["meta"][f"{name}/K{k}"]
    o = oracle.ref_pdhg(lp, max_iterations=k)
    assert o["status"] == meta["status"]
    assert o["iterations"] == meta["iterations"]
    assert np.array_equal(o["y_last"], golden["arrays"][f"{name}/K{k}/y"])
    assert lp.n == len(golden["arrays"][f"{name}/K{k}/x"])  # no presolve reduction on these
    assert np.array_equal(o["x_final"], golden["arrays"][f"{name}/K{k}/x"])
    assert o["constraint_violation"] == meta["constraint_violation"]
    assert o["bound_violation"] == meta["bound_violation"]


@pytest.mark.parametrize("case", [c for c in fo_cases.CASES], ids=[c[0] for c in fo_cases.CASES])
def test_oracle_matches_reference_known_answers(oracle, golden, golden_std, case):
    name, _, lp, exp = case
    meta = golden["meta"][name]
    if meta["sf_status"] != 0:
        pytest.skip("reference solved this case in presolve (no PDHG iterations)")
    std = golden_std(name)
    o = oracle.ref_pdhg(std, max_iterations=meta["max_iterations"])
    assert o["status"] == meta["status"]
    assert o["iterations"] == meta["iterations"]
    assert np.array_equal(o["y_last"], golden["arrays"][f"{name}/y"])


def test_oracle_live_reference_fresh_seeds(oracle, reflib, lpgen):
    for seed in (101, 202):
        lp = lpgen.random_sparse(m=50, n=140, nnz_per_col=3, seed=seed)
        sf = reflib.standard_form(lp)
        try:
            assert sf["status"] == 0

            class S:
                pass
            s = S()
            for f in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub", "is_eq"):
                setattr(s, f, sf[f])
            s.m, s.n = sf["m"], sf["n"]
            for k in (3, 250, 2000):
                r = reflib.fo_solve(lp, max_iterations=k)
                o = oracle.ref_pdhg(s, max_iterations=k)
                assert r["status"] == o["status"] and r["iterations"] == o["iterations"]
                assert np.array_equal(r["y"], o["y_last"])
                x, obj = reflib.recover(sf, o["x_final"])
                assert np.array_equal(r["x"], x)
                assert r["objective"] == obj
        finally:
            reflib.free(sf)


def test_oracle_spmv_matches_reference(oracle, reflib, lpgen):
    lp = lpgen.random_sparse(m=80, n=200, nnz_per_col=4, seed=3).standard()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(lp.n)
    y = rng.standard_normal(lp.m)
    assert np.array_equal(oracle.spmv(lp, x), reflib.spmv(lp.m, lp.n, lp.rowptr, lp.colidx, lp.vals, x))
    assert np.array_equal(oracle.spmv_t(lp, y), reflib.spmv_t(lp.m, lp.n, lp.rowptr, lp.colidx, lp.vals, y))


def test_known_answer_values(golden):
    """The reference's own answers satisfy the assertions of its tests (the golden file is sane)."""
    for name, _, lp, exp in fo_cases.CASES:
        meta = golden["meta"][name]
        if exp["status"] == "NOT_OPTIMAL":
            assert meta["status"] != "OPTIMAL"
            continue
        assert meta["status"] == exp["status"], name
        x = golden["arrays"][f"{name}/x"]
        for j, (v, tol) in exp.get("x", {}).items():
            assert abs(x[j] - v) <= tol, (name, j, x[j], v)
        if "obj" in exp:
            assert abs(meta["objective"] - exp["obj"][0]) <= exp["obj"][1], name
        if "iterations" in exp:
            assert meta["iterations"] == exp["iterations"]


def test_kkt_checker_at_highs_optimum(golden, lpgen):
    import scipy.sparse as sp
    from scipy.optimize import linprog

    import pdlp_oracle
    lp = lpgen.random_sparse(m=40, n=120, nnz_per_col=3, seed=11).standard()
    A = sp.csr_matrix((lp.vals, lp.colidx, lp.rowptr), shape=(lp.m, lp.n))
    eq = lp.is_eq.astype(bool)
    r = linprog(lp.c, A_ub=A[~eq], b_ub=lp.b[~eq], A_eq=A[eq], b_eq=lp.b[eq], bounds=list(zip(lp.lb, lp.ub)),
                method="highs")
    assert abs(r.fun - golden["highs"]["rs_small"]) <= 1e-9 * max(1, abs(r.fun))
    # HiGHS duals use the opposite sign convention (d obj / d b); the reference Lagrangian is c.x + y.(Ax-b)
    y = np.zeros(lp.m)
    y[~eq] = -r.ineqlin.marginals
    y[eq] = -r.eqlin.marginals
    k = pdlp_oracle.kkt(lp, r.x, y)
    assert k["rel_kkt"] < 1e-9, k


def test_restated_engine_reaches_highs(golden, lpgen):
    import pdlp_oracle
    lp = lpgen.random_sparse(m=40, n=120, nnz_per_col=3, seed=11).standard()
    x, y, info = pdlp_oracle.halpern_pdhg(lp, eps=1e-7)
    assert info["status"] == "OPTIMAL"
    z = golden["highs"]["rs_small"]
    assert abs(info["pobj"] - z) <= 1e-6 * max(1.0, abs(z))
