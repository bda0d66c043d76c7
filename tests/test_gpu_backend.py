"""GpuBackend primitives on the GPU (the cases of the reference's
tests/test_gpu_foundation.cpp:58-323), checked bit for bit against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def csr(m, n, entries):
    entries = sorted(entries)
    rowptr = np.zeros(m + 1, np.int32)
    for r, _, _ in entries:
        rowptr[r + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, np.array([e[1] for e in entries], np.int32), np.array([e[2] for e in entries], np.float64)


CASES = {
    "identity": (3, 3, [(0, 0, 1.0), (1, 1, 1.0), (2, 2, 1.0)], [5.0, -3.0, 7.0], [5.0, -3.0, 7.0]),
    "diagonal": (3, 3, [(0, 0, 2.0), (1, 1, 4.0), (2, 2, 8.0)], [1.0, 2.0, 3.0], [2.0, 8.0, 24.0]),
    "small_sparse": (2, 3, [(0, 0, 1.0), (0, 2, 2.0), (1, 1, 3.0)], [4.0, 5.0, 6.0], [16.0, 15.0]),
    "rectangular": (4, 2, [(0, 0, 1.0), (1, 1, 2.0), (2, 0, 3.0), (3, 1, 4.0)], [10.0, 20.0], [10.0, 40.0, 30.0, 80.0]),
    "dense2x2": (2, 2, [(0, 0, 3.0), (0, 1, 4.0), (1, 0, 1.0), (1, 1, 2.0)], [2.0, 3.0], [18.0, 8.0]),
    "tiny_values": (1, 1, [(0, 0, 1e-8)], [1e-8], [1e-16]),
}


@pytest.mark.parametrize("name", list(CASES))
def test_spmv_known_answers(ctx, name):
    m, n, ent, x, want = CASES[name]
    rp, ci, va = csr(m, n, ent)
    y, timing = ctx.spmv(m, n, rp, ci, va, np.array(x))
    assert np.array_equal(y, np.array(want)) or np.allclose(y, want, rtol=0, atol=1e-18)
    assert all(v >= 0.0 for v in timing.values())


def test_spmv_banded_and_large_diagonal(ctx, oracle):
    ent = [(i, i, float(i + 1)) for i in range(10)] + [(i, i + 1, 0.5) for i in range(9)]
    rp, ci, va = csr(10, 10, ent)
    y, _ = ctx.spmv(10, 10, rp, ci, va, np.ones(10))
    assert np.array_equal(y, np.array([float(i + 1) + (0.5 if i < 9 else 0.0) for i in range(10)]))
    rp, ci, va = csr(1000, 1000, [(i, i, 2.0) for i in range(1000)])
    y, _ = ctx.spmv(1000, 1000, rp, ci, va, np.full(1000, 3.0))
    assert np.all(y == 6.0)


@pytest.mark.parametrize("seed,m,n,k", [(0, 300, 1000, 5), (1, 20000, 100000, 8), (2, 7, 3, 2)])
def test_spmv_and_transpose_bit_exact(ctx, oracle, lpgen, seed, m, n, k):
    lp = lpgen.random_sparse(m=m, n=n, nnz_per_col=k, seed=seed).standard()
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n)
    y = rng.standard_normal(m)
    gy, _ = ctx.spmv(m, n, lp.rowptr, lp.colidx, lp.vals, x)
    gw, _ = ctx.spmv(m, n, lp.rowptr, lp.colidx, lp.vals, y, transpose=True)
    assert np.array_equal(gy, oracle.spmv(lp, x))
    assert np.array_equal(gw, oracle.spmv_t(lp, y))


def test_spmv_invalid_arguments(ctx, b2p):
    # empty matrix -> INVALID_ARGUMENT (test_gpu_foundation.cpp:265-269)
    with pytest.raises(b2p.B2PError) as e:
        ctx.spmv(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), np.zeros(0))
    assert e.value.code == b2p.INVALID_ARGUMENT
    # unsorted / out-of-range column indices are rejected, not computed
    rp, ci, va = np.array([0, 2], np.int32), np.array([1, 0], np.int32), np.array([1.0, 2.0])
    with pytest.raises(b2p.B2PError) as e:
        ctx.spmv(1, 2, rp, ci, va, np.ones(2))
    assert e.value.code == b2p.INVALID_ARGUMENT
    ci = np.array([0, 5], np.int32)
    with pytest.raises(b2p.B2PError) as e:
        ctx.spmv(1, 2, rp, ci, va, np.ones(2))
    assert e.value.code == b2p.INVALID_ARGUMENT


def test_vector_ops(ctx):
    a = np.array([1.0, 2.0, 3.0])
    b = np.array([4.0, 5.0, 6.0])
    assert np.array_equal(ctx.vector_op("add", a, b), [5.0, 7.0, 9.0])
    assert np.array_equal(ctx.vector_op("sub", a, b), [-3.0, -3.0, -3.0])
    assert np.array_equal(ctx.vector_op("scale", np.array([2.0, 4.0, 6.0]), alpha=2.5), [5.0, 10.0, 15.0])
    assert np.array_equal(ctx.vector_op("axpy", a, np.array([10.0, 20.0, 30.0]), alpha=3.0), [13.0, 26.0, 39.0])
    assert ctx.dot(a, b) == 32.0
    assert ctx.norm2(np.array([3.0, 4.0, 0.0])) == 5.0


def test_reductions_large(ctx):
    rng = np.random.default_rng(5)
    a = rng.standard_normal(3_000_001)
    b = rng.standard_normal(3_000_001)
    assert abs(ctx.dot(a, b) - float(a @ b)) <= 1e-12 * float(np.abs(a) @ np.abs(b))
    assert abs(ctx.norm2(a) - float(np.linalg.norm(a))) <= 1e-13 * float(np.linalg.norm(a))
    # deterministic: same inputs, same bits
    assert ctx.dot(a, b) == ctx.dot(a, b)


def test_device_info(b2p):
    info = b2p.device_info(0)
    assert info["is_available"] and info["cc"] == (10, 0)
    assert info["sm_count"] >= 100 and info["total_memory_bytes"] > 100 * 2**30
