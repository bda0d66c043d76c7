"""Known-answer LPs of the reference's first-order solver tests, as data.

Each case restates the model built in tests/test_first_order_solver.cpp of the
reference (file:line given per case) and the values that test asserts.  The
same cases drive the oracle pinning tests (CPU) and the GPU engine tests.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parents[2] / "mangalore-refinery-and-petrochemicals-limited_b200"
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))
import lpgen  # noqa: E402

INF = math.inf
LE, EQ, GE = lpgen.LE, lpgen.EQ, lpgen.GE


def make_lp(name, maximize, variables, constraints):
    """variables: list of (lb, ub, obj); constraints: list of (terms {j: a}, sense, rhs)."""
    n = len(variables)
    m = len(constraints)
    rowptr = [0]
    colidx, vals = [], []
    for terms, _, _ in constraints:
        for j in sorted(terms):
            colidx.append(j)
            vals.append(terms[j])
        rowptr.append(len(colidx))
    return lpgen.LP(m, n, np.array(rowptr, np.int32), np.array(colidx, np.int32), np.array(vals, np.float64),
                    np.array([c[1] for c in constraints], np.int32), np.array([c[2] for c in constraints], np.float64),
                    np.array([v[2] for v in variables], np.float64), np.array([v[0] for v in variables], np.float64),
                    np.array([v[1] for v in variables], np.float64), maximize, name)


# (name, reference test line, lp, expected): expected keys -- status ("OPTIMAL" or "NOT_OPTIMAL"),
# obj (value, tol), x {index: (value, tol)}, iterations (exact)
CASES = [
    ("FO_01_one_var_bounded", "test_first_order_solver.cpp:10-21",
     make_lp("fo01", False, [(2.0, 5.0, 3.0)], []),
     {"status": "OPTIMAL", "x": {0: (2.0, 1e-3)}, "obj": (6.0, 1e-3)}),
    ("FO_02_two_var_simple", "test_first_order_solver.cpp:23-35",
     make_lp("fo02", True, [(0, 10, 2.0), (0, 10, 3.0)], [({0: 1.0, 1: 1.0}, LE, 6.0)]),
     {"status": "OPTIMAL", "obj": (18.0, 1e-2)}),
    ("FO_03_equality", "test_first_order_solver.cpp:37-50",
     make_lp("fo03", False, [(0, 10, 1.0), (0, 10, 2.0)], [({0: 1.0, 1: 1.0}, EQ, 4.0)]),
     {"status": "OPTIMAL", "obj": (4.0, 1e-3), "xsum": (4.0, 1e-3)}),
    ("FO_04_greater_than", "test_first_order_solver.cpp:52-64",
     make_lp("fo04", False, [(0, 10, 4.0)], [({0: 1.0}, GE, 3.0)]),
     {"status": "OPTIMAL", "x": {0: (3.0, 1e-3)}, "obj": (12.0, 1e-3)}),
    ("FO_05_mixed", "test_first_order_solver.cpp:66-80",
     make_lp("fo05", True, [(0, 10, 3.0), (0, 10, 5.0)], [({0: 1.0, 1: 1.0}, LE, 8.0), ({0: 1.0}, GE, 1.0)]),
     {"status": "OPTIMAL", "obj": (38.0, 1e-2)}),
    ("FO_06_lower_bound", "test_first_order_solver.cpp:82-92",
     make_lp("fo06", False, [(3.0, INF, 2.0)], []),
     {"status": "OPTIMAL", "x": {0: (3.0, 1e-3)}}),
    ("FO_07_upper_bound", "test_first_order_solver.cpp:94-104",
     make_lp("fo07", True, [(0.0, 7.0, 5.0)], []),
     {"status": "OPTIMAL", "x": {0: (7.0, 1e-3)}}),
    ("FO_08_doubly_bounded", "test_first_order_solver.cpp:106-116",
     make_lp("fo08", False, [(-2.0, 4.0, 3.0)], []),
     {"status": "OPTIMAL", "x": {0: (-2.0, 1e-3)}}),
    ("FO_09_free_variable", "test_first_order_solver.cpp:118-129",
     make_lp("fo09", False, [(-INF, INF, 1.0)], [({0: 1.0}, GE, -5.0)]),
     {"status": "OPTIMAL", "x": {0: (-5.0, 1e-2)}}),
    ("FO_10_fixed_variable", "test_first_order_solver.cpp:131-142",
     make_lp("fo10", True, [(4.0, 4.0, 5.0)], []),
     {"status": "OPTIMAL", "x": {0: (4.0, 1e-3)}, "obj": (20.0, 1e-3)}),
    ("FO_11_zero_objective", "test_first_order_solver.cpp:144-155",
     make_lp("fo11", False, [(0.0, 5.0, 0.0)], [({0: 1.0}, GE, 2.0)]),
     {"status": "OPTIMAL", "obj": (0.0, 1e-3)}),
    ("FO_12_redundant", "test_first_order_solver.cpp:157-170",
     make_lp("fo12", True, [(0.0, 10.0, 4.0)], [({0: 1.0}, LE, 5.0), ({0: 1.0}, LE, 8.0)]),
     {"status": "OPTIMAL", "x": {0: (5.0, 1e-3)}}),
    ("FO_13_degenerate", "test_first_order_solver.cpp:172-185",
     make_lp("fo13", True, [(0, 10, 2.0), (0, 10, 3.0)], [({0: 1.0, 1: 1.0}, LE, 0.0)]),
     {"status": "OPTIMAL", "obj": (0.0, 1e-3)}),
    ("FO_14_small_coefficients", "test_first_order_solver.cpp:187-198",
     make_lp("fo14", False, [(0.0, 10.0, 1e-4)], [({0: 1e-4}, GE, 1e-3)]),
     {"status": "OPTIMAL", "x": {0: (10.0, 1e-2)}}),
    ("FO_15_mixed_scales", "test_first_order_solver.cpp:200-213",
     make_lp("fo15", True, [(0, 10, 100.0), (0, 10, 1.0)], [({0: 10.0, 1: 0.1}, LE, 50.0)]),
     {"status": "OPTIMAL", "obj": (500.0, 1e-2)}),
    ("FO_16_presolve_reduced", "test_first_order_solver.cpp:215-229",
     make_lp("fo16", True, [(3.0, 3.0, 2.0), (0.0, 10.0, 4.0)], [({0: 1.0, 1: 1.0}, LE, 8.0)]),
     {"status": "OPTIMAL", "x": {0: (3.0, 1e-3), 1: (5.0, 1e-2)}}),
    ("FO_17_rectangular", "test_first_order_solver.cpp:231-245",
     make_lp("fo17", False, [(0, 10, 1.0), (0, 10, 2.0), (0, 10, 3.0)], [({0: 1.0, 1: 1.0}, GE, 4.0)]),
     {"status": "OPTIMAL", "obj": (4.0, 1e-2)}),
    ("FO_18_larger_sparse", "test_first_order_solver.cpp:247-266",
     make_lp("fo18", True, [(0.0, 5.0, 1.0)] * 20, [({i: 1.0, i + 10: 1.0}, LE, 6.0) for i in range(10)]),
     {"status": "OPTIMAL", "obj": (60.0, 1e-1)}),
    ("FO_19_hand_lp", "test_first_order_solver.cpp:268-286",
     make_lp("fo19", True, [(0.0, INF, 3.0), (0.0, INF, 5.0)], [({0: 2.0, 1: 1.0}, LE, 8.0), ({0: 1.0, 1: 2.0}, LE, 8.0)]),
     {"status": "OPTIMAL", "x": {0: (8.0 / 3.0, 1e-2), 1: (8.0 / 3.0, 1e-2)}, "obj": (64.0 / 3.0, 1e-2)}),
    ("FO_20_infeasible_bounds", "test_first_order_solver.cpp:288-297",
     make_lp("fo20", False, [(5.0, 2.0, 1.0)], []),
     {"status": "NOT_OPTIMAL"}),
    ("FO_22_verifier", "test_first_order_solver.cpp:311-323",
     make_lp("fo22", True, [(0.0, 10.0, 4.0)], [({0: 1.0}, LE, 6.0)]),
     {"status": "OPTIMAL", "verified": True}),
    ("FO_23_cpu_vs_gpu", "test_first_order_solver.cpp:325-345",
     make_lp("fo23", True, [(0, 10, 2.0), (0, 10, 3.0)], [({0: 1.0, 1: 1.0}, LE, 5.0)]),
     {"status": "OPTIMAL"}),
    ("FO_25_iteration_limit", "test_first_order_solver.cpp:361-375",
     make_lp("fo25", True, [(0, 100, 5.0), (0, 100, 6.0)], [({0: 1.0, 1: 1.0}, LE, 50.0)]),
     {"status": "MAX_ITERATIONS", "iterations": 5, "max_iterations": 5}),
]
