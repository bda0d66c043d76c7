"""ORACLE -- test infrastructure only (never imported by the product path).

1. ``kkt``: FP64 relative-KKT evaluator for the standard-form LP
       min c.x  s.t.  (Ax)_i <= b_i (is_eq=0) / = b_i (is_eq=1),  lb <= x <= ub
   with the Lagrangian of the reference PDHG (src/first_order_solver.cpp:185-192:
   y_i >= 0 on <= rows, L = c.x + y.(Ax - b)).  Definitions follow PDLP
   (Applegate et al. 2021): primal residual ||(Ax-b)_proj||_2, dual residual
   ||c + A^T y - lambda||_2 with lambda the bound multipliers, duality gap
   |c.x - (-b.y + sum l lambda+ - u lambda-)|; relative to 1+||b||, 1+||c||,
   1+|p|+|d|.

2. ``ruiz_pc_scaling`` / ``power_norm`` / ``halpern_pdhg``: FP64 numpy
   restatement of the engine algorithm the CUDA path implements (restarted
   Halpern PDHG with reflection, Lu & Yang 2024 "Restarted Halpern PDHG for
   linear programming"; Ruiz + Pock-Chambolle diagonal scaling; PDLP primal
   weight smoothing).  The reference has no counterpart for this algorithm;
   its parity is pinned by the FP64 KKT above, by HiGHS objectives and by the
   reference's SolutionVerifier (src/solution_verifier.cpp:42-204).
"""
from __future__ import annotations

import numpy as np


def _rows(lp):
    return np.repeat(np.arange(lp.m), np.diff(lp.rowptr))


def spmv(lp, x):
    return np.bincount(_rows(lp), weights=lp.vals * x[lp.colidx], minlength=lp.m)


def spmv_t(lp, y):
    return np.bincount(lp.colidx, weights=lp.vals * y[_rows(lp)], minlength=lp.n)


def kkt(lp, x, y, eps=None):
    """FP64 KKT components of (x, y) on the standard-form LP. Returns a dict."""
    b, c, lb, ub = lp.b, lp.c, lp.lb, lp.ub
    eq = lp.is_eq.astype(bool)
    ax = spmv(lp, x)
    rp = ax - b
    rp = np.where(eq, rp, np.maximum(rp, 0.0))
    # dual feasibility of y: y >= 0 on <= rows; a negative y there is a dual violation
    yv = np.where(eq, 0.0, np.minimum(y, 0.0))
    g = c + spmv_t(lp, y)
    fl, fu = np.isfinite(lb), np.isfinite(ub)
    lam = np.where(fl & fu, g, np.where(fl, np.maximum(g, 0.0), np.where(fu, np.minimum(g, 0.0), 0.0)))
    rd = g - lam
    pobj = float(c @ x)
    dobj = float(-b @ y + np.sum(np.where(lam > 0, lam * np.where(fl, lb, 0.0), 0.0))
                 + np.sum(np.where(lam < 0, lam * np.where(fu, ub, 0.0), 0.0)))
    out = {
        "primal_res": float(np.linalg.norm(rp)),
        "dual_res": float(np.sqrt(np.linalg.norm(rd) ** 2 + np.linalg.norm(yv) ** 2)),
        "pobj": pobj,
        "dobj": dobj,
        "gap": abs(pobj - dobj),
        "bnorm": float(np.linalg.norm(b)),
        "cnorm": float(np.linalg.norm(c)),
    }
    out["rel_primal"] = out["primal_res"] / (1.0 + out["bnorm"])
    out["rel_dual"] = out["dual_res"] / (1.0 + out["cnorm"])
    out["rel_gap"] = out["gap"] / (1.0 + abs(pobj) + abs(dobj))
    out["rel_kkt"] = max(out["rel_primal"], out["rel_dual"], out["rel_gap"])
    if eps is not None:
        out["converged"] = out["rel_kkt"] <= eps
    return out


def ruiz_pc_scaling(lp, ruiz_iters=10):
    """Ruiz l-inf equilibration then Pock-Chambolle (alpha=1) column/row scaling.
    Returns (dr, dc) with A_s = diag(dr) A diag(dc)."""
    rows = _rows(lp)
    a = np.abs(lp.vals)
    dr = np.ones(lp.m)
    dc = np.ones(lp.n)
    for _ in range(ruiz_iters):
        s = a * dr[rows] * dc[lp.colidx]
        rmax = np.zeros(lp.m)
        np.maximum.at(rmax, rows, s)
        cmax = np.zeros(lp.n)
        np.maximum.at(cmax, lp.colidx, s)
        dr = dr / np.sqrt(np.where(rmax > 0, rmax, 1.0))
        dc = dc / np.sqrt(np.where(cmax > 0, cmax, 1.0))
    s = a * dr[rows] * dc[lp.colidx]
    rsum = np.bincount(rows, weights=s, minlength=lp.m)
    csum = np.bincount(lp.colidx, weights=s, minlength=lp.n)
    dr = dr / np.sqrt(np.where(rsum > 0, rsum, 1.0))
    dc = dc / np.sqrt(np.where(csum > 0, csum, 1.0))
    return dr, dc


def scaled(lp, dr, dc):
    from copy import copy
    s = copy(lp)
    s.vals = lp.vals * dr[_rows(lp)] * dc[lp.colidx]
    s.b = lp.b * dr
    s.c = lp.c * dc
    s.lb = lp.lb / dc
    s.ub = lp.ub / dc
    return s


def power_norm(lp, iters=100, seed=0, tol=1e-7):
    """Largest singular value of A by power iteration on A^T A."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(lp.n)
    v /= np.linalg.norm(v)
    sig = 0.0
    for _ in range(iters):
        w = spmv_t(lp, spmv(lp, v))
        nw = np.linalg.norm(w)
        if nw == 0:
            return 0.0
        new = np.sqrt(nw)
        v = w / nw
        if abs(new - sig) <= tol * new:
            sig = new
            break
        sig = new
    return sig


def halpern_pdhg(lp, eps=1e-6, max_iter=100000, check_every=64, reflect=1.0, x0=None, y0=None, omega0=None,
                 beta_suff=0.2, beta_nec=0.8, beta_art=0.36, step_safety=0.998, dtype=np.float64,
                 ruiz_iters=10, verbose=False):
    """Restarted Halpern PDHG with reflection on the scaled LP; KKT checked in FP64 on the
    original LP every `check_every` iterations. Returns (x, y, info)."""
    dr, dc = ruiz_pc_scaling(lp, ruiz_iters)
    s = scaled(lp, dr, dc)
    eta = step_safety / power_norm(s)
    cn, bn = np.linalg.norm(s.c), np.linalg.norm(s.b)
    omega = omega0 if omega0 is not None else (cn / bn if cn > 1e-10 and bn > 1e-10 else 1.0)
    eq = s.is_eq.astype(bool)
    # values and iterates are STORED in `dtype`; sums and updates are computed in FP64
    A32 = s.vals.astype(dtype).astype(np.float64)
    rows = _rows(s)

    def Ax(v):
        return np.bincount(rows, weights=A32 * v.astype(np.float64)[s.colidx], minlength=s.m)

    def ATy(v):
        return np.bincount(s.colidx, weights=A32 * v.astype(np.float64)[rows], minlength=s.n)

    c = s.c.astype(dtype).astype(np.float64); b = s.b.astype(dtype).astype(np.float64)
    l = s.lb.astype(dtype).astype(np.float64); u = s.ub.astype(dtype).astype(np.float64)
    x = (np.clip(np.zeros(s.n), s.lb, s.ub) if x0 is None else np.clip(x0 / dc, s.lb, s.ub)).astype(dtype)
    y = (np.zeros(s.m) if y0 is None else y0 / dr).astype(dtype)
    if y0 is not None:
        y = np.where(eq, y, np.maximum(y, 0)).astype(dtype)
    xa, ya = x.copy(), y.copy()
    k = 0
    total = 0
    r0 = None
    rprev = None
    restarts = 0
    info = {}
    while total < max_iter:
        tau, sigma = eta / omega, eta * omega
        x64, y64 = x.astype(np.float64), y.astype(np.float64)
        xt = np.clip(x64 - tau * (c + ATy(y)), l, u)
        xh = (2 * xt - x64).astype(dtype)
        yt = y64 + sigma * (Ax(xh) - b)
        yt = np.where(eq, yt, np.maximum(yt, 0))
        check = (k == 0) or ((total + 1) % check_every == 0)
        if check:
            r = np.sqrt(omega * np.sum((x - xt).astype(np.float64) ** 2) + np.sum((y - yt).astype(np.float64) ** 2) / omega)
        # Halpern step with reflection
        w = (k + 1.0) / (k + 2.0)
        x = (w * ((1 + reflect) * xt - reflect * x64) + (1 - w) * xa.astype(np.float64)).astype(dtype)
        y = (w * ((1 + reflect) * yt - reflect * y64) + (1 - w) * ya.astype(np.float64)).astype(dtype)
        xt = xt.astype(dtype)
        yt = yt.astype(dtype)
        k += 1
        total += 1
        if not check:
            continue
        if k == 1:
            r0 = r
            rprev = r
            if total % check_every != 0:
                continue
        # termination on the original problem
        kk = kkt(lp, xt.astype(np.float64) * dc, yt.astype(np.float64) * dr)
        if verbose and total % (check_every * 50) == 0:
            print(total, restarts, omega, kk["rel_primal"], kk["rel_dual"], kk["rel_gap"])
        if kk["rel_kkt"] <= eps:
            info.update(kk)
            info.update(iterations=total, restarts=restarts, status="OPTIMAL", omega=omega)
            return xt.astype(np.float64) * dc, yt.astype(np.float64) * dr, info
        restart = (r <= beta_suff * r0) or (r <= beta_nec * r0 and r > rprev) or (k >= beta_art * total)
        rprev = r
        if restart:
            dx = np.linalg.norm((xt - xa).astype(np.float64))
            dy = np.linalg.norm((yt - ya).astype(np.float64))
            if dx > 1e-10 and dy > 1e-10:
                omega = float(np.exp(0.5 * np.log(dy / dx) + 0.5 * np.log(omega)))
            x, y = xt.copy(), yt.copy()
            xa, ya = xt.copy(), yt.copy()
            k = 0
            restarts += 1
    kk = kkt(lp, xt.astype(np.float64) * dc, yt.astype(np.float64) * dr)
    info.update(kk)
    info.update(iterations=total, restarts=restarts, status="MAX_ITERATIONS", omega=omega)
    return xt.astype(np.float64) * dc, yt.astype(np.float64) * dr, info
