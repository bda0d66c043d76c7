"""The benchmark's full-size workloads on the GPU, checked with the oracle's FP64 KKT.

* block-angular blending LP (m = 204,000, n = 1,000,000, 8.0M nonzeros): single-LP
  engine, mixed precision and FP64, to 1e-6 relative KKT;
* 4,096 uneven LPs (m ~ logU(50, 2000)) in one batched solve, every answer checked;
* ill-conditioned stress LP (m = 1M, n = 5M, 50M nonzeros): a capped mixed solve
  (the full solve to 1e-8 takes minutes), checking that the FP64 KKT the engine
  evaluates on the device agrees with the oracle's on the returned answer -- the
  stop decision at full size rests on that number.
"""
from __future__ import annotations

import numpy as np
import pytest

import pdlp_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def block_angular(lpgen):
    return lpgen.block_angular().standard()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_block_angular_full_size(ctx, block_angular, precision):
    s = block_angular
    ctx.upload(s)
    res, x, y = ctx.solve(engine="halpern", precision=precision, eps=1e-6, max_iterations=100000)
    assert res["status"] == "OPTIMAL", res
    k = pdlp_oracle.kkt(s, x, y)
    assert k["rel_kkt"] <= 1.05e-6, k
    assert abs(res["primal_objective"] - k["pobj"]) <= 1e-9 * max(1.0, abs(k["pobj"]))


def test_uneven_batch_full_size(ctx, lpgen):
    lps = lpgen.uneven_batch()
    stds = [lp.standard() for lp in lps]
    mats = [(s.m, s.n, s.rowptr, s.colidx, s.vals) for s in stds]
    ctx.batch_upload(mats, np.arange(len(stds), dtype=np.int32), np.concatenate([s.b for s in stds]),
                     np.concatenate([s.c for s in stds]), np.concatenate([s.lb for s in stds]),
                     np.concatenate([s.ub for s in stds]), np.concatenate([s.is_eq for s in stds]))
    _, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-6, eps_objective=1e-6, max_iterations=400000)
    assert np.all(per["status"] == 0), np.bincount(per["status"])
    obj = ctx.batch_objectives()
    xo = np.cumsum([0] + [s.n for s in stds])
    yo = np.cumsum([0] + [s.m for s in stds])
    worst = 0.0
    for i, s in enumerate(stds):
        k = pdlp_oracle.kkt(s, x[xo[i]:xo[i + 1]], y[yo[i]:yo[i + 1]])
        worst = max(worst, k["rel_kkt"])
        assert abs(obj["pobj"][i] - k["pobj"]) <= 1e-9 * max(1.0, abs(k["pobj"])), i
    assert worst <= 1.05e-6, worst
    assert np.all(obj["obj_err"] <= 1e-6)


def test_ill_conditioned_full_size_kkt_agrees(ctx, lpgen):
    s = lpgen.ill_conditioned().standard()
    ctx.upload(s)
    res, x, y = ctx.solve(engine="halpern", precision="fp32", eps=1e-8, max_iterations=4096)
    assert res["status"] == "MAX_ITERATIONS", res
    k = pdlp_oracle.kkt(s, x, y)
    for dev, ora in (("rel_primal_residual", "rel_primal"), ("rel_dual_residual", "rel_dual"), ("rel_gap", "rel_gap")):
        assert res[dev] == pytest.approx(k[ora], rel=1e-6, abs=1e-14), (dev, res[dev], k[ora])
    assert res["primal_objective"] == pytest.approx(k["pobj"], rel=1e-9)
