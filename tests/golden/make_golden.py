"""Generates tests/golden/ref_traces.npz and tests/golden/highs_objectives.json.

Run in a container that has the reference tree (it loads the reference's own
code compiled by `make -C oracle ref`):

    python tests/golden/make_golden.py

* For every known-answer case of tests/golden/fo_cases.py and for seeded
  random LPs, it records what the reference CPUFirstOrderSolver returns
  (status, iterations, objective, primal and dual vectors) -- including runs
  cut at small max_iterations, whose dual vector is the reference iterate y^K.
* It records the reference's presolved standard form of each case, so the GPU
  tests can feed exactly what the reference PDHG iterated on.
* It records scipy-HiGHS optimal objectives of the seeded LPs used by the
  Halpern-engine tests (exact-objective oracle).
The outputs are small and committed; the GPU tests read only these files.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests" / "golden"))
sys.path.insert(0, str(ROOT / "mangalore-refinery-and-petrochemicals-limited_b200"))

import fo_cases  # noqa: E402
import lpgen  # noqa: E402
from oracle_lib import RefLib  # noqa: E402


def seeded_lps():
    """Small seeded LPs whose reference traces are pinned."""
    return {
        "rs_c0": lpgen.random_sparse(),                       # the 300 x 1000 workload
        "rs_small": lpgen.random_sparse(m=40, n=120, nnz_per_col=3, seed=11),
        "rs_ge": lpgen.block_angular(periods=2, block_rows=30, block_cols=90, nnz_per_col=3, link_rows=10, seed=5),
    }


def highs_objective(std):
    import scipy.sparse as sp
    from scipy.optimize import linprog
    A = sp.csr_matrix((std.vals, std.colidx, std.rowptr), shape=(std.m, std.n))
    eq = std.is_eq.astype(bool)
    r = linprog(std.c, A_ub=A[~eq] if (~eq).any() else None, b_ub=std.b[~eq] if (~eq).any() else None,
                A_eq=A[eq] if eq.any() else None, b_eq=std.b[eq] if eq.any() else None,
                bounds=list(zip(std.lb, std.ub)), method="highs")
    assert r.status == 0, r.message
    return float(r.fun)


def highs_lps():
    out = {
        "rs_c0": lpgen.random_sparse(),
        "rs_small": lpgen.random_sparse(m=40, n=120, nnz_per_col=3, seed=11),
        "ba_mini": lpgen.block_angular(periods=5, block_rows=400, block_cols=2000, link_rows=400),
        "ba_tiny": lpgen.block_angular(periods=3, block_rows=60, block_cols=300, nnz_per_col=4, link_rows=30, seed=9),
        "ill_small": lpgen.ill_conditioned(m=300, n=1500, nnz_per_col=4, seed=4),
    }
    for i, lp in enumerate(lpgen.uneven_batch(6, seed=12)):
        out[f"batch12_{i}"] = lp
    fam = lpgen.RefineryFamily()
    out["refinery_p0"] = fam.instance(fam.sample_params(1, 0)[0])
    plan = lpgen.RefineryPlanningFamily()
    for i, q in enumerate(plan.sample_params(3, 20001)):  # the first held-out instances of the benchmark
        out[f"planning_heldout_{i}"] = plan.instance(q)
    return out


def main():
    ref = RefLib()
    arrays = {}
    meta = {}
    for name, line, lp, exp in fo_cases.CASES:
        kmax = exp.get("max_iterations", 50000)
        r = ref.fo_solve(lp, max_iterations=kmax)
        key = name
        arrays[f"{key}/x"] = r["x"]
        arrays[f"{key}/y"] = r["y"]
        meta[key] = {"status": r["status"], "iterations": r["iterations"], "objective": r["objective"],
                     "max_iterations": kmax, "source": line}
        sf = ref.standard_form(lp)
        meta[key]["sf_status"] = sf["status"]
        if sf["status"] == 0:
            for f in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub", "is_eq"):
                arrays[f"{key}/sf_{f}"] = sf[f]
        ref.free(sf)
    for name, lp in seeded_lps().items():
        sf = ref.standard_form(lp)
        assert sf["status"] == 0
        for f in ("rowptr", "colidx", "vals", "b", "c", "lb", "ub", "is_eq"):
            arrays[f"{name}/sf_{f}"] = sf[f]
        ref.free(sf)
        for k in (1, 7, 100, 1000):
            r = ref.fo_solve(lp, max_iterations=k)
            arrays[f"{name}/K{k}/x"] = r["x"]
            arrays[f"{name}/K{k}/y"] = r["y"]
            meta[f"{name}/K{k}"] = {"status": r["status"], "iterations": r["iterations"], "objective": r["objective"],
                                    "constraint_violation": r["constraint_violation"],
                                    "bound_violation": r["bound_violation"]}
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_traces.npz", **arrays)
    (ROOT / "tests" / "golden" / "ref_traces.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    hi = {name: highs_objective(lp.standard()) for name, lp in highs_lps().items()}
    (ROOT / "tests" / "golden" / "highs_objectives.json").write_text(json.dumps(hi, indent=1, sort_keys=True))
    print(f"wrote {len(arrays)} arrays, {len(meta)} reference records, {len(hi)} HiGHS objectives")


if __name__ == "__main__":
    main()
