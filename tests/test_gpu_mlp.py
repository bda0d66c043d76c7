"""Tensor-core GEMM and the warm-start MLP on the GPU, against the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,ta,tb", [(128, 128, 64, False, False), (256, 1024, 256, False, True),
                                         (200, 300, 100, True, False), (256, 10001, 1024, False, True),
                                         (10001, 64, 256, True, True), (8, 8, 8, False, False),
                                         (1000, 520, 4100, False, False)])
def test_gemm_bf16_exact_to_fp32_accumulation(ctx, M, N, K, ta, tb):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
    B = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
    Ab, Bb = mo.bf16_bits(A), mo.bf16_bits(B)
    C = ctx.gemm_bf16(Ab, Bb, trans_a=ta, trans_b=tb)
    Af, Bf = mo.bf16(A), mo.bf16(B)
    Am = Af.T if ta else Af
    Bm = Bf.T if tb else Bf
    ref = Am @ Bm
    bound = np.abs(Am) @ np.abs(Bm)
    err = np.abs(C - ref)
    assert np.all(err <= 2e-6 * bound + 1e-30), (err.max(), (err / (bound + 1e-30)).max())


def test_mlp_gradient_matches_oracle(ctx):
    i, h, o, n = 64, 128, 40, 48
    rng = np.random.default_rng(5)
    ctx.mlp_create(i, h, o, seed=3)
    flat = (rng.standard_normal(ctx.mlp_param_count()) * 0.1).astype(np.float32)
    ctx.mlp_set_params(flat)
    assert np.array_equal(ctx.mlp_get_params(), flat)
    X = rng.standard_normal((n, i)).astype(np.float32)
    T = rng.standard_normal((n, o)).astype(np.float32)
    loss, g = ctx.mlp_gradient(X, T)
    loss_ref, grads = mo.loss_and_grad(flat, X.astype(np.float64), T.astype(np.float64), i, h, o)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    s = 0
    for name, gr in zip(("W1", "b1", "W2", "b2", "W3", "b3"), grads):
        gg = g[s:s + gr.size].reshape(gr.shape)
        s += gr.size
        rel = np.linalg.norm(gg - gr) / max(np.linalg.norm(gr), 1e-30)
        assert rel <= 2e-2, (name, rel)


def test_mlp_inference_matches_oracle(ctx):
    i, h, o, n = 256, 1024, 10001, 300
    rng = np.random.default_rng(9)
    ctx.mlp_create(i, h, o, seed=11)
    flat = ctx.mlp_get_params()
    X = rng.uniform(-1, 1, (n, i)).astype(np.float32)
    Y = ctx.mlp_infer(X)
    Yref = mo.forward(flat, X.astype(np.float64), i, h, o)[-1]
    rel = np.linalg.norm(Y - Yref) / np.linalg.norm(Yref)
    assert rel <= 2e-2, rel


def test_mlp_training_reduces_loss(ctx):
    i, h, o, n = 64, 256, 32, 2048
    rng = np.random.default_rng(1)
    P = rng.standard_normal((i, o)) / np.sqrt(i)
    X = rng.uniform(-1, 1, (n, i)).astype(np.float32)
    T = np.tanh(X @ P).astype(np.float32)
    ctx.mlp_create(i, h, o, seed=2)
    losses = [ctx.mlp_train_epoch(X, T, batch=128, lr=2e-3) for _ in range(40)]
    assert losses[-1] < 0.1 * losses[0], losses[::8]


def test_mlp_gradient_split_k_matches_oracle(ctx):
    """Hidden width 1024 and 1000 outputs on 64 rows: the 1024-deep hidden layer and the
    output-gradient GEMM (K = 1000) fill few output tiles and run split along K; the
    gradients still match the FP64 oracle to BF16 rounding."""
    i, h, o, n = 256, 1024, 1000, 64
    rng = np.random.default_rng(15)
    ctx.mlp_create(i, h, o, seed=4)
    flat = (rng.standard_normal(ctx.mlp_param_count()) * 0.03).astype(np.float32)
    ctx.mlp_set_params(flat)
    X = rng.standard_normal((n, i)).astype(np.float32)
    T = rng.standard_normal((n, o)).astype(np.float32)
    loss, g = ctx.mlp_gradient(X, T)
    loss_ref, grads = mo.loss_and_grad(flat, X.astype(np.float64), T.astype(np.float64), i, h, o)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    s = 0
    for name, gr in zip(("W1", "b1", "W2", "b2", "W3", "b3"), grads):
        gg = g[s:s + gr.size].reshape(gr.shape)
        s += gr.size
        rel = np.linalg.norm(gg - gr) / max(np.linalg.norm(gr), 1e-30)
        assert rel <= 2e-2, (name, rel)


def test_mlp_device_training_is_deterministic(ctx, lpgen, b2p):
    """b2p_mlp_train replays one captured epoch graph: two runs from the same seed on the
    same device data set end with bit-identical parameters and a lower loss than after
    one epoch."""
    fam = lpgen.RefineryFamily()
    P = fam.sample_params(24, 5)
    b2p.warmstart.upload_family(ctx, fam, P)
    ctx.batch_solve(precision="fp32", eps=1e-5, outputs=False)
    params = []
    for _ in range(2):
        ctx.mlp_create(fam.N_PARAM, 256, fam.n + fam.m + 1, seed=7)
        ctx.mlp_dataset_from_batch(P.astype(np.float32))
        first = ctx.mlp_train(1, batch=8, lr_start=1e-3, lr_end=1e-3, seed=3)
        last = ctx.mlp_train(6, batch=8, lr_start=1e-3, lr_end=1e-4, seed=3)
        assert last < first
        params.append(ctx.mlp_get_params())
    assert np.array_equal(params[0], params[1])
