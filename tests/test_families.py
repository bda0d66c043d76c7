"""Workload generators (CPU): shapes, determinism and the batched standard form of
the parametric refinery families."""
from __future__ import annotations

import numpy as np


def test_planning_family_structure(lpgen):
    fam = lpgen.RefineryPlanningFamily()
    assert (fam.m, fam.n) == (2000, 8000)
    nnz = int(fam.rowptr[-1])
    assert 5.9 <= nnz / fam.n <= 6.1  # 6 nonzeros per column on average
    assert np.all(np.isfinite(fam.ub)) and np.all(fam.lb == 0)  # every column boxed -> bounded
    again = lpgen.RefineryPlanningFamily()
    np.testing.assert_array_equal(fam.vals, again.vals)  # seed-fixed structure
    P = fam.sample_params(64, 20001)
    assert P.shape == (64, 256)
    assert np.all((P[:, :128] >= 0.8) & (P[:, :128] <= 1.2)) and np.all((P[:, 128:] >= 0.7) & (P[:, 128:] <= 1.3))
    narrow = fam.sample_params(64, 20001, spread=0.05)
    np.testing.assert_allclose(narrow - 1.0, 0.05 * (P - 1.0))


def test_standard_batch_matches_per_instance_standard_form(lpgen):
    for fam in (lpgen.RefineryPlanningFamily(), lpgen.RefineryFamily()):
        P = fam.sample_params(3, 7)
        s0, B, Cc, LB, UB, EQ = fam.standard_batch(P)
        for i, q in enumerate(P):
            s = fam.instance(q).standard()
            np.testing.assert_array_equal(s.rowptr, s0.rowptr)
            np.testing.assert_array_equal(s.vals, s0.vals)
            np.testing.assert_array_equal(s.b, B[i])
            np.testing.assert_array_equal(s.c, Cc[i])
            np.testing.assert_array_equal(s.lb, LB[i])
            np.testing.assert_array_equal(s.ub, UB[i])
            np.testing.assert_array_equal(s.is_eq, EQ[i])


def test_parameters_move_prices_and_rhs(lpgen):
    fam = lpgen.RefineryPlanningFamily()
    one = np.ones(256)
    c1, b1 = fam.costs(one), fam.rhs(one)
    np.testing.assert_allclose(c1, fam.base_cost)
    np.testing.assert_allclose(b1, fam.rhs_base)
    p = one.copy()
    p[3] = 1.1  # crude-price group 3
    moved = np.flatnonzero(fam.costs(p) != c1)
    assert len(moved) > 0 and np.all(fam.cpar_kind[moved] == 1)
    p = one.copy()
    p[192] = 1.2  # demand scale group 0
    moved = np.flatnonzero(fam.rhs(p) != b1)
    assert len(moved) > 0 and np.all(fam.sense[moved] == lpgen.GE)
