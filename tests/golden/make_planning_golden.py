"""Generates tests/golden/planning_heldout_highs.json: scipy-HiGHS optimal
objectives of the first 64 held-out instances of the benchmark's refinery
planning family (lpgen.RefineryPlanningFamily, held-out parameter seed 20001).

The GPU tests check the batched engine's answers at the benchmark's stop
criterion against these values with the max(1, |z|) denominator of the
reference's docs/testing-strategy.md:56.  HiGHS is the one bundled with scipy
(an exact simplex / IPM optimum); nothing here needs the reference tree.

    python tests/golden/make_planning_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests" / "golden"))
sys.path.insert(0, str(ROOT / "mangalore-refinery-and-petrochemicals-limited_b200"))

import lpgen  # noqa: E402
from make_golden import highs_objective  # noqa: E402

COUNT = 64
SEED = 20001


def main():
    fam = lpgen.RefineryPlanningFamily()
    P = fam.sample_params(COUNT, SEED)
    out = {"seed": SEED, "count": COUNT, "objectives": []}
    for q in P:
        out["objectives"].append(highs_objective(fam.instance(q).standard()))
    (ROOT / "tests" / "golden" / "planning_heldout_highs.json").write_text(json.dumps(out, indent=1))
    print(f"wrote {COUNT} HiGHS objectives")


if __name__ == "__main__":
    main()
