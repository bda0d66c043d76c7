"""Infeasibility and unboundedness certificates, single-LP and batched engines.

The reference's status enum has INFEASIBLE_DETECTED and UNBOUNDED_DETECTED
(include/bharatopt/first_order_solver.hpp:15-22) but its PDHG only reports
infeasibility that presolve finds (src/first_order_solver.cpp:28-34; the
FO_20 / FO_21 cases of tests/test_first_order_solver.cpp:288-309).  The engines
here certify both from the fixed-point displacement T(z) - z (a dual ray for an
infeasible LP, a primal ray for an unbounded one), as branch-and-bound needs to
prune infeasible nodes.  The checker of each case's true status is scipy's
HiGHS; feasible instances in the same batch must still come back OPTIMAL with
the oracle's FP64 KKT within tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linprog

import pdlp_oracle

pytestmark = pytest.mark.gpu


def _with_rows(lpgen, std, rows, b, eq):
    """std plus extra rows (dense list of {col: value}), standard form."""
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n)).tolil()
    A.resize((std.m + len(rows), std.n))
    for k, r in enumerate(rows):
        for j, v in r.items():
            A[std.m + k, j] = v
    A = A.tocsr()
    A.sort_indices()
    return lpgen.StdLP(A.shape[0], A.shape[1], A.indptr.astype(np.int32), A.indices.astype(np.int32),
                       A.data.astype(np.float64), np.concatenate([std.b, b]), std.c.copy(), std.lb.copy(),
                       std.ub.copy(), np.concatenate([std.is_eq, np.array(eq, np.uint8)]), name="rows")


def _with_col(lpgen, std, entries, c, lb, ub):
    """std plus one extra column (rows -> value)."""
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n)).tolil()
    A.resize((std.m, std.n + 1))
    for i, v in entries.items():
        A[i, std.n] = v
    A = A.tocsr()
    A.sort_indices()
    return lpgen.StdLP(A.shape[0], A.shape[1], A.indptr.astype(np.int32), A.indices.astype(np.int32),
                       A.data.astype(np.float64), std.b.copy(), np.append(std.c, c), np.append(std.lb, lb),
                       np.append(std.ub, ub), std.is_eq.copy(), name="col")


def _highs_status(std):
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n))
    eq = std.is_eq.astype(bool)
    r = linprog(std.c, A_ub=A[~eq] if (~eq).any() else None, b_ub=std.b[~eq] if (~eq).any() else None,
                A_eq=A[eq] if eq.any() else None, b_eq=std.b[eq] if eq.any() else None,
                bounds=list(zip(std.lb, [None if np.isinf(u) else u for u in std.ub])), method="highs")
    return {0: "OPTIMAL", 2: "INFEASIBLE_DETECTED", 3: "UNBOUNDED_DETECTED"}[r.status]


def cases(lpgen):
    """(name, standard-form LP, expected status)."""
    out = []
    base = lpgen.random_sparse(m=60, n=200, nnz_per_col=3, seed=21).standard()
    out.append(("feasible", base, "OPTIMAL"))
    # 40 boxed [0, 10] columns cannot sum to 500: infeasible through the bounds
    out.append(("infeasible_eq_sum", _with_rows(lpgen, base, [{j: 1.0 for j in range(40)}], [500.0], [1]),
                "INFEASIBLE_DETECTED"))
    # sum_S x <= 1 and sum_S x >= 5: two contradictory inequalities
    S = {j: 1.0 for j in range(3, 60, 3)}
    out.append(("infeasible_pair", _with_rows(lpgen, base, [S, {j: -v for j, v in S.items()}], [1.0, -5.0], [0, 0]),
                "INFEASIBLE_DETECTED"))
    # a free-above column with cost -1 whose entries only relax <= rows: unbounded
    le_rows = [i for i in range(base.m) if not base.is_eq[i]][:4]
    out.append(("unbounded_col", _with_col(lpgen, base, {i: -1.0 for i in le_rows}, -1.0, 0.0, np.inf),
                "UNBOUNDED_DETECTED"))
    return out


@pytest.fixture(scope="module")
def all_cases(lpgen):
    cs = cases(lpgen)
    for name, std, exp in cs:
        assert _highs_status(std) == exp, name  # the checker agrees with the construction
    return cs


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_single_lp_certificates(ctx, all_cases, precision):
    for name, std, exp in all_cases:
        ctx.upload(std)
        res, x, y = ctx.solve(engine="halpern", precision=precision, eps=1e-6, max_iterations=200000)
        assert res["status"] == exp, (name, res["status"], res["iterations"])
        if exp == "OPTIMAL":
            assert pdlp_oracle.kkt(std, x, y)["rel_kkt"] <= 1.05e-6


def test_single_lp_certificates_off(ctx, all_cases):
    """eps_infeasible = 0 turns detection off: the infeasible LP runs to the cap."""
    name, std, exp = all_cases[1]
    ctx.upload(std)
    res, _, _ = ctx.solve(engine="halpern", precision="fp64", eps=1e-6, max_iterations=4096, eps_infeasible=0.0)
    assert res["status"] == "MAX_ITERATIONS"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_certificates_mixed_batch(ctx, all_cases, precision):
    """Feasible, infeasible and unbounded instances in one batched launch: each gets
    its own status; the feasible ones are solved to tolerance."""
    stds = [std for _, std, _ in all_cases] * 2
    exps = [exp for _, _, exp in all_cases] * 2
    mats = [(s.m, s.n, s.rowptr, s.colidx, s.vals) for s in stds]
    ctx.batch_upload(mats, np.arange(len(stds), dtype=np.int32), np.concatenate([s.b for s in stds]),
                     np.concatenate([s.c for s in stds]), np.concatenate([s.lb for s in stds]),
                     np.concatenate([s.ub for s in stds]), np.concatenate([s.is_eq for s in stds]))
    _, per, x, y = ctx.batch_solve(precision=precision, eps=1e-6, max_iterations=200000)
    names = ["OPTIMAL", "MAX_ITERATIONS", "NUMERICAL_FAILURE", "INFEASIBLE_DETECTED", "UNBOUNDED_DETECTED"]
    got = [names[s] for s in per["status"]]
    assert got == exps, (got, per["iterations"])
    xo = np.cumsum([0] + [s.n for s in stds])
    yo = np.cumsum([0] + [s.m for s in stds])
    for i, s in enumerate(stds):
        if exps[i] == "OPTIMAL":
            k = pdlp_oracle.kkt(s, x[xo[i]:xo[i + 1]], y[yo[i]:yo[i + 1]])
            assert k["rel_kkt"] <= 1.05e-6, (i, k)


def test_feasible_family_has_no_false_certificates(ctx, lpgen):
    """Sixty-four feasible uneven LPs with certificates on: every one OPTIMAL."""
    lps = lpgen.uneven_batch(64, m_hi=400, seed=23)
    stds = [lp.standard() for lp in lps]
    mats = [(s.m, s.n, s.rowptr, s.colidx, s.vals) for s in stds]
    ctx.batch_upload(mats, np.arange(len(stds), dtype=np.int32), np.concatenate([s.b for s in stds]),
                     np.concatenate([s.c for s in stds]), np.concatenate([s.lb for s in stds]),
                     np.concatenate([s.ub for s in stds]), np.concatenate([s.is_eq for s in stds]))
    _, per, _, _ = ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=200000, outputs=False)
    assert np.all(per["status"] == 0), per["status"]
