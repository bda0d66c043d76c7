"""Learned warm start for a parametric LP family sharing one constraint matrix.

Sequences the device-side steps exposed by the C ABI; no solution data crosses
to the host on the training path:

1. labels: the batched engine solves N training instances to `label_eps`
   relative KKT (b2p_batch_solve; answers stay on the device);
2. data set: b2p_mlp_dataset_from_batch builds normalised inputs (the parameter
   vectors) and targets [x, y, log primal weight] on the device;
3. training: b2p_mlp_train runs Adam on the BF16 tcgen05 forward / backward
   kernels, reshuffling every epoch, cosine learning-rate decay;
4. solving: b2p_batch_solve_learned predicts x0, y0 and the primal weight on the
   device, solves warm-started and re-solves cold every instance the warm run
   did not solve (cold-start fallback).

The family object provides ``N_PARAM``, ``sample_params(count, seed)`` and
``standard_batch(P)`` (shared standard-form matrix and per-instance b, c, l, u,
row kinds), as ``lpgen.RefineryPlanningFamily`` does.
"""
from __future__ import annotations

import time

import numpy as np


def upload_family(ctx, family, P):
    """Uploads the instances of parameter vectors P (count x N_PARAM) as one batch
    sharing the family's matrix; returns the shared standard-form matrix."""
    s0, B, Cc, LB, UB, EQ = family.standard_batch(P)
    count = B.shape[0]
    ctx.batch_upload([(s0.m, s0.n, s0.rowptr, s0.colidx, s0.vals)], np.zeros(count, np.int32), B.ravel(), Cc.ravel(),
                     LB.ravel(), UB.ravel(), EQ.ravel().astype(np.uint8))
    return s0


class LearnedWarmStart:
    """MLP N_PARAM -> hidden -> hidden -> (n + m + 1) trained on the method's own answers."""

    def __init__(self, ctx, family, hidden: int = 1024, seed: int = 0):
        self.ctx, self.family, self.hidden, self.seed = ctx, family, hidden, seed
        self.stats = {}

    def fit(self, n_train: int = 20000, label_eps: float = 1e-8, epochs: int = 200, batch: int = 1024,
            lr: float = 2e-3, param_seed: int = 1, max_iterations: int = 1_000_000):
        ctx, fam = self.ctx, self.family
        P = fam.sample_params(n_train, param_seed)
        t0 = time.perf_counter()
        s0 = upload_family(ctx, fam, P)
        summ, per, _, _ = ctx.batch_solve(precision="fp32", eps=label_eps, max_iterations=max_iterations,
                                          outputs=False)
        t1 = time.perf_counter()
        ctx.mlp_create(fam.N_PARAM, self.hidden, s0.n + s0.m + 1, seed=self.seed)
        ctx.mlp_dataset_from_batch(P.astype(np.float32))
        loss = ctx.mlp_train(epochs, batch=batch, lr_start=lr, lr_end=lr * 1e-2, seed=self.seed)
        t2 = time.perf_counter()
        self.stats = {"n_train": n_train, "label_eps": label_eps, "label_s": t1 - t0,
                      "label_solved": int((per["status"] == 0).sum()),
                      "label_iterations_mean": float(per["iterations"].mean()), "epochs": epochs, "batch": batch,
                      "train_s": t2 - t1, "train_loss": loss}
        return self.stats

    def solve(self, P, eps: float = 1e-6, fallback: bool = True, precision: str = "fp32",
              max_iterations: int = 1_000_000, outputs: bool = True, upload: bool = True,
              eps_objective: float = 0.0):
        """Learned-warm batched solve of the instances of P (uploads them unless
        upload=False, when they are already the context's batch).  eps_objective > 0
        also asks each answer's objective to be within that relative distance of the
        optimum (b2p_params.eps_objective)."""
        if upload:
            upload_family(self.ctx, self.family, P)
        return self.ctx.batch_solve_learned(np.asarray(P, np.float32), fallback=fallback, precision=precision,
                                            eps=eps, eps_objective=eps_objective, max_iterations=max_iterations,
                                            outputs=outputs)
