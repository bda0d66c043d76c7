"""ORACLE -- test infrastructure only.

FP64 numpy restatement of the warm-start MLP (in -> hidden -> hidden -> out,
tanh-form GELU, mean-squared error), rounding to BF16 exactly where the GPU
path stores BF16: the input, the weights, the two hidden activations, the
output gradient and the two hidden gradients.  Accumulation is FP64 here (FP32
on the tensor cores), so GPU gradients agree to BF16/FP32 rounding.  The
reference has no learned component; this oracle pins the tensor-core forward
and backward instead.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def bf16_bits(x):
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


K = 0.7978845608028654


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K * (1.0 + 3 * 0.044715 * x * x)


def unflatten(flat, i, h, o):
    s = 0
    out = []
    for shape in ((h, i), (h,), (h, h), (h,), (o, h), (o,)):
        n = int(np.prod(shape))
        out.append(np.asarray(flat[s:s + n], np.float64).reshape(shape))
        s += n
    return out


def forward(flat, X, i, h, o):
    W1, b1, W2, b2, W3, b3 = unflatten(flat, i, h, o)
    Xb = bf16(X)
    Z1 = Xb @ bf16(W1).T + b1
    H1 = bf16(gelu(Z1))
    Z2 = H1 @ bf16(W2).T + b2
    H2 = bf16(gelu(Z2))
    Y = H2 @ bf16(W3).T + b3
    return Xb, Z1, H1, Z2, H2, Y


def loss_and_grad(flat, X, T, i, h, o):
    W1, b1, W2, b2, W3, b3 = unflatten(flat, i, h, o)
    Xb, Z1, H1, Z2, H2, Y = forward(flat, X, i, h, o)
    n = X.shape[0]
    loss = float(np.mean((Y - T) ** 2))
    dY = bf16(2.0 * (Y - T) / (n * o))
    gW3 = dY.T @ H2
    gb3 = dY.sum(0)
    dH2 = dY @ bf16(W3)
    dZ2 = bf16(dH2 * gelu_grad(Z2))
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(0)
    dH1 = dZ2 @ bf16(W2)
    dZ1 = bf16(dH1 * gelu_grad(Z1))
    gW1 = dZ1.T @ Xb
    gb1 = dZ1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]
