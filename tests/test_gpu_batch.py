"""Batched engine on the GPU: many independent LPs in one persistent launch.

Every instance's answer is checked by the oracle's FP64 KKT; objectives of the
instances with committed HiGHS values are checked to 1e-6 relative."""
from __future__ import annotations

import numpy as np
import pytest

import pdlp_oracle

pytestmark = pytest.mark.gpu


def upload_lps(ctx, lps):
    stds = [lp.standard() for lp in lps]
    mats = [(s.m, s.n, s.rowptr, s.colidx, s.vals) for s in stds]
    ctx.batch_upload(mats, np.arange(len(stds), dtype=np.int32), np.concatenate([s.b for s in stds]),
                     np.concatenate([s.c for s in stds]), np.concatenate([s.lb for s in stds]),
                     np.concatenate([s.ub for s in stds]), np.concatenate([s.is_eq for s in stds]))
    return stds


def split(stds, x, y):
    xo = np.cumsum([0] + [s.n for s in stds])
    yo = np.cumsum([0] + [s.m for s in stds])
    return [(x[xo[i]:xo[i + 1]], y[yo[i]:yo[i + 1]]) for i in range(len(stds))]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_uneven_all_optimal(ctx, golden, lpgen, precision):
    lps = lpgen.uneven_batch(6, seed=12) + lpgen.uneven_batch(58, m_hi=600, seed=13)
    stds = upload_lps(ctx, lps)
    summ, per, x, y = ctx.batch_solve(precision=precision, eps=1e-6, max_iterations=100000)
    assert np.all(per["status"] == 0), per["status"]
    for i, (s, (xi, yi)) in enumerate(zip(stds, split(stds, x, y))):
        k = pdlp_oracle.kkt(s, xi, yi)
        assert k["rel_kkt"] <= 1.05e-6, (i, k)
        assert abs(k["rel_kkt"] - per["rel_kkt"][i]) <= 1e-8 + 1e-3 * k["rel_kkt"]
        if i < 6:
            z = golden["highs"][f"batch12_{i}"]
            assert abs(k["pobj"] - z) <= 1e-6 * max(1.0, abs(z)), (i, k["pobj"], z)


def test_batch_mixed_refinement_tight(ctx, golden, lpgen):
    """FP32 matrix values with FP64 re-centring at every restart reach 1e-9 rel KKT."""
    lps = lpgen.uneven_batch(6, seed=12) + lpgen.uneven_batch(10, m_hi=500, seed=14)
    stds = upload_lps(ctx, lps)
    summ, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-9, max_iterations=200000)
    assert np.all(per["status"] == 0), (per["status"], per["iterations"])
    assert np.all(np.isfinite(per["omega"])) and np.all(per["omega"] > 0)
    for i, (s, (xi, yi)) in enumerate(zip(stds, split(stds, x, y))):
        k = pdlp_oracle.kkt(s, xi, yi)
        assert k["rel_kkt"] <= 1.05e-9, (i, k)
        if i < 6:
            z = golden["highs"][f"batch12_{i}"]
            assert abs(k["pobj"] - z) <= 1e-8 * max(1.0, abs(z)), (i, k["pobj"], z)


def test_batch_matches_single_engine(ctx, lpgen):
    lps = lpgen.uneven_batch(4, seed=31)
    stds = upload_lps(ctx, lps)
    _, per, x, y = ctx.batch_solve(precision="fp64", eps=1e-8, max_iterations=200000)
    for s, (xi, yi) in zip(stds, split(stds, x, y)):
        k = pdlp_oracle.kkt(s, xi, yi)
        ctx.upload(s)
        res, xs, ys = ctx.solve(engine="halpern", precision="fp64", eps=1e-8, max_iterations=200000)
        assert res["status"] == "OPTIMAL"
        assert abs(k["pobj"] - res["primal_objective"]) <= 1e-7 * max(1.0, abs(k["pobj"]))


def test_batch_shared_matrix_family(ctx, golden, lpgen):
    fam = lpgen.RefineryFamily()
    p = np.vstack([fam.sample_params(1, 0), fam.sample_params(15, 77)])
    inst = [fam.instance(q) for q in p]
    stds = [lp.standard() for lp in inst]
    s0 = stds[0]
    ctx.batch_upload([(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals)], np.zeros(len(stds), np.int32),
                     np.concatenate([s.b for s in stds]), np.concatenate([s.c for s in stds]),
                     np.concatenate([s.lb for s in stds]), np.concatenate([s.ub for s in stds]),
                     np.concatenate([s.is_eq for s in stds]))
    _, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=200000)
    assert np.all(per["status"] == 0)
    for i, (s, (xi, yi)) in enumerate(zip(stds, split(stds, x, y))):
        k = pdlp_oracle.kkt(s, xi, yi)
        assert k["rel_kkt"] <= 1.05e-6
    z = golden["highs"]["refinery_p0"]
    k0 = pdlp_oracle.kkt(stds[0], *split(stds, x, y)[0])
    assert abs(k0["pobj"] - z) <= 1e-6 * abs(z)


def test_batch_warm_start_and_weights(ctx, lpgen):
    lps = lpgen.uneven_batch(8, m_hi=400, seed=40)
    stds = upload_lps(ctx, lps)
    _, per, x, y = ctx.batch_solve(precision="fp64", eps=1e-7)
    cold = per["iterations"].copy()
    _, per2, x2, y2 = ctx.batch_solve(x0=x, y0=y, precision="fp64", eps=1e-6)
    assert np.all(per2["status"] == 0)
    assert np.all(per2["iterations"] <= 128), (cold, per2["iterations"])


def test_batch_iteration_limit(ctx, lpgen):
    lps = lpgen.uneven_batch(5, m_hi=300, seed=41)
    upload_lps(ctx, lps)
    _, per, _, _ = ctx.batch_solve(precision="fp32", eps=1e-12, max_iterations=256)
    assert np.all(per["status"] == 1) and np.all(per["iterations"] == 256)


def test_batch_rejects_bad_input(ctx, b2p):
    rp = np.array([0, 2], np.int32)
    ci = np.array([1, 0], np.int32)  # not ascending
    with pytest.raises(b2p.B2PError) as e:
        ctx.batch_upload([(1, 2, rp, ci, np.ones(2))], np.zeros(1, np.int32), np.ones(1), np.ones(2), np.zeros(2),
                         np.ones(2), np.zeros(1, np.uint8))
    assert e.value.code == b2p.INVALID_ARGUMENT


def test_planning_family_matches_highs(ctx, golden, lpgen, b2p):
    """The first held-out instances of the benchmark's refinery planning family:
    mixed-precision batched answers at 1e-9 relative KKT reach the HiGHS optimum to
    1e-6 relative.  (Every column is boxed and the duals are O(1e3) against
    ||b|| ~ 2e3, so the objective of an answer at relative KKT eps can be off by
    ~200 eps relative: 2e-6 at 1e-8.)"""
    fam = lpgen.RefineryPlanningFamily()
    P = fam.sample_params(3, 20001)
    s0, B, Cc, LB, UB, EQ = fam.standard_batch(P)
    b2p.warmstart.upload_family(ctx, fam, P)
    _, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-9, max_iterations=1000000)
    assert np.all(per["status"] == 0), per
    for i in range(3):
        s = lpgen.StdLP(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals, B[i], Cc[i], LB[i], UB[i], EQ[i])
        k = pdlp_oracle.kkt(s, x[i * fam.n:(i + 1) * fam.n], y[i * fam.m:(i + 1) * fam.m])
        assert k["rel_kkt"] <= 1.05e-9, (i, k)
        z = golden["highs"][f"planning_heldout_{i}"]
        assert abs(k["pobj"] - z) <= 1e-6 * max(1.0, abs(z)), (i, k["pobj"], z)


def test_batch_instance_too_large_is_an_error(ctx, lpgen, b2p):
    """A batched instance whose y and xh do not fit one CTA's shared memory (here
    30,000 x 60,000 in FP32: 360 KB) is refused with INVALID_ARGUMENT, not run."""
    lp = lpgen.random_sparse(m=30000, n=60000, nnz_per_col=2, seed=3).standard()
    ctx.batch_upload([(lp.m, lp.n, lp.rowptr, lp.colidx, lp.vals)], np.zeros(1, np.int32), lp.b, lp.c, lp.lb, lp.ub,
                     lp.is_eq)
    with pytest.raises(b2p.B2PError) as e:
        ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=1000, outputs=False)
    assert e.value.code == b2p.INVALID_ARGUMENT
    assert "shared memory" in str(e.value)


def _planning_check(per, x, y, fam, P, s0, B, Cc, LB, UB, EQ, lpgen, reflib, zs, eps):
    """Every answer counted as solved (status OPTIMAL): FP64 relative KKT <= eps
    (oracle), objective within eps of the HiGHS optimum with the max(1, |z|)
    denominator of the reference's docs/testing-strategy.md:56, and the reference
    SolutionVerifier accepts x at the absolute feasibility tolerance eps (1 + ||b||)
    that a relative primal residual of eps allows.

    The rest stop at the iteration cap (MAX_ITERATIONS) and are not counted.  On
    this sample that is at most 3 of 64 (instances 0, 9 and 28: the oracle's own
    FP64 Halpern PDHG stalls on the same three, its relative gap still 3e-6 to 4e-4
    after 400,000 iterations with the primal residual below 1e-9)."""
    assert np.all((per["status"] == 0) | (per["status"] == 1)), per["status"]
    assert int((per["status"] == 0).sum()) >= len(P) - 3, (per["status"], per["iterations"])
    for i in range(len(P)):
        if per["status"][i] != 0:
            continue
        s = lpgen.StdLP(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals, B[i], Cc[i], LB[i], UB[i], EQ[i])
        xi, yi = x[i * fam.n:(i + 1) * fam.n], y[i * fam.m:(i + 1) * fam.m]
        k = pdlp_oracle.kkt(s, xi, yi)
        assert k["rel_kkt"] <= 1.05 * eps, (i, k)
        assert abs(k["pobj"] - zs[i]) <= eps * max(1.0, abs(zs[i])), (i, k["pobj"], zs[i])
        lp = fam.instance(P[i])
        v = reflib.verify(lp, xi, feas_tol=eps * (1 + float(np.linalg.norm(B[i]))), reported_obj=float(lp.obj @ xi))
        assert v["verified"] == 1, (i, v)


def test_planning_heldout_answers_cold(ctx, lpgen, b2p, reflib):
    """The benchmark's stop criterion (relative KKT 1e-6 and the device's objective-error
    bound 1e-6) on its first 64 held-out instances, mixed precision from the cold
    start: every counted answer passes the FP64 checks."""
    import json
    from conftest import GOLDEN
    g = json.loads((GOLDEN / "planning_heldout_highs.json").read_text())
    fam = lpgen.RefineryPlanningFamily()
    P = fam.sample_params(g["count"], g["seed"])
    s0, B, Cc, LB, UB, EQ = fam.standard_batch(P)
    b2p.warmstart.upload_family(ctx, fam, P)
    _, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-6, eps_objective=1e-6, max_iterations=400000)
    objs = ctx.batch_objectives()
    solved = per["status"] == 0
    assert np.all(objs["obj_err"][solved] <= 1e-6)
    # a capped instance reports that its criterion does not hold
    assert np.all((per["rel_kkt"][~solved] > 1e-6) | (objs["obj_err"][~solved] > 1e-6))
    _planning_check(per, x, y, fam, P, s0, B, Cc, LB, UB, EQ, lpgen, reflib, g["objectives"], 1e-6)


def test_planning_heldout_answers_learned(ctx, lpgen, b2p, reflib):
    """The same 64 instances learned-warm (a small model: 512 labels to 1e-8, 30 epochs)
    at the benchmark's stop criterion: every counted warm-started answer passes the FP64 checks."""
    import json
    from conftest import GOLDEN
    g = json.loads((GOLDEN / "planning_heldout_highs.json").read_text())
    fam = lpgen.RefineryPlanningFamily()
    ws = b2p.warmstart.LearnedWarmStart(ctx, fam)
    ws.fit(n_train=512, label_eps=1e-8, epochs=30, max_iterations=400000)
    P = fam.sample_params(g["count"], g["seed"])
    s0, B, Cc, LB, UB, EQ = fam.standard_batch(P)
    summ, per, x, y = ws.solve(P, eps=1e-6, eps_objective=1e-6, max_iterations=400000)
    _planning_check(per, x, y, fam, P, s0, B, Cc, LB, UB, EQ, lpgen, reflib, g["objectives"], 1e-6)


def test_batch_autotuned_shape(ctx, lpgen, tmp_path, monkeypatch):
    """The batched autotuner picks the CTA size and the chunk length (iterations per
    persistent launch, a power of two in [256, 8192] whose fixed cost is <= 2 % of its
    iterations); the summary reports threads * 1e5 + chunk, and a second solve of the
    same precision reuses the tuned shape."""
    monkeypatch.setenv("B2P_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    lps = lpgen.uneven_batch(40, m_hi=500, seed=44)
    upload_lps(ctx, lps)
    summ, per, _, _ = ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=100000, outputs=False)
    threads, chunk = divmod(int(round(summ["step_size"])), 100000)
    assert threads in (128, 256, 512)
    assert 256 <= chunk <= 8192 and chunk & (chunk - 1) == 0
    assert np.all(per["status"] == 0)
    summ2, per2, _, _ = ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=100000, outputs=False)
    assert summ2["step_size"] == summ["step_size"]
    assert np.array_equal(per2["iterations"], per["iterations"])  # deterministic


def test_batch_trace_and_objectives(ctx, lpgen):
    """The active-instance trace of a solve runs from the batch size down to zero in
    increasing time, and the per-instance objectives agree with the oracle's."""
    lps = lpgen.uneven_batch(24, m_hi=400, seed=45)
    stds = upload_lps(ctx, lps)
    _, per, x, y = ctx.batch_solve(precision="fp64", eps=1e-7, max_iterations=200000)
    t, active = ctx.batch_trace()
    assert active[0] == len(stds) and active[-1] == 0
    assert np.all(np.diff(active) <= 0) and np.all(np.diff(t) >= 0)
    obj = ctx.batch_objectives()
    for i, (s, (xi, yi)) in enumerate(zip(stds, split(stds, x, y))):
        k = pdlp_oracle.kkt(s, xi, yi)
        assert abs(obj["pobj"][i] - k["pobj"]) <= 1e-9 * max(1.0, abs(k["pobj"]))
        assert abs(obj["dobj"][i] - k["dobj"]) <= 1e-6 * max(1.0, abs(k["dobj"]))
        assert np.isfinite(obj["obj_err"][i]) and obj["obj_err"][i] >= 0.0


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_pair_form_matches_single(b2p, lpgen, tmp_path, monkeypatch, precision):
    """The paired form (two instances of the shared matrix per CTA, each SELL load
    feeding both instances' gathers) reproduces the single form bit for bit at the
    same CTA size and entry order: statuses, iteration counts and answers.  63
    planning instances, so one CTA holds an unpaired instance, and pairs part when one
    member finishes first."""
    monkeypatch.setenv("B2P_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    fam = lpgen.RefineryPlanningFamily()
    P = fam.sample_params(63, 777)
    out = {}
    forms = (1, 2)
    for ni in forms:
        monkeypatch.setenv("B2P_BATCH_SHAPE", f"256,2,{ni}")
        c = b2p.Context(0)
        try:
            b2p.warmstart.upload_family(c, fam, P)
            summ, per, x, y = c.batch_solve(precision=precision, eps=1e-5, max_iterations=30000)
            assert int(round(summ["used_average"])) == 10 * ni + 2
            assert int(round(summ["step_size"])) // 100000 == 256
            out[ni] = (per, x, y)
        finally:
            c.close()
    p1, x1, y1 = out[1]
    assert len(set(p1["iterations"].tolist())) > 1  # instances finish at different iterations
    for ni in forms[1:]:
        p2, x2, y2 = out[ni]
        assert np.array_equal(p1["status"], p2["status"]), ni
        assert np.array_equal(p1["iterations"], p2["iterations"]), ni
        assert np.array_equal(x1, x2) and np.array_equal(y1, y2), ni


def test_batch_pair_form_chosen_only_for_shared_matrix(ctx, lpgen, tmp_path, monkeypatch):
    """A pinned paired shape on a batch of different matrices runs one instance per CTA."""
    monkeypatch.setenv("B2P_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    monkeypatch.setenv("B2P_BATCH_SHAPE", "256,1,2")
    stds = upload_lps(ctx, lpgen.uneven_batch(12, m_hi=300, seed=46))
    summ, per, x, y = ctx.batch_solve(precision="fp32", eps=1e-6, max_iterations=100000)
    assert int(round(summ["used_average"])) == 11
    assert np.all(per["status"] == 0)
    for s, (xi, yi) in zip(stds, split(stds, x, y)):
        assert pdlp_oracle.kkt(s, xi, yi)["rel_kkt"] <= 1.05e-6
