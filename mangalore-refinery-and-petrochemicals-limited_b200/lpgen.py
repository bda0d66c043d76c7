"""Seeded synthetic LP families used by the tests and the benchmark.

Every instance is produced in the reference's *original* row form (senses
<=, =, >=; the shape of ``LPModel``, include/bharatopt/lp_model.hpp:50-127)
and can be converted to the standard form the reference PDHG iterates on
(``A x (<= | =) b``, >= rows negated; src/first_order_solver.cpp:68-101) with
:meth:`LP.standard`.

Families (sizes as named by the workload they stand for):

* :func:`random_sparse`   -- m=300 (150 =, 150 <=), n=1000, 5 nnz per column.
* :func:`block_angular`   -- 50 period blocks of 4000 x 20000 (8 nnz/col,
  lognormal values with random sign) linked by 4000 inventory-balance rows.
* :func:`uneven_batch`    -- 4096 independent LPs, m ~ logU(50, 2000),
  n = m * U(2, 5), 4-10 nnz per column.
* :class:`RefineryFamily` -- fixed 2000 x 8000 structure (6 nnz/col), a
  256-dimensional parameter vector scales prices and rhs.
* :func:`ill_conditioned` -- m=1M, n=5M, 10 nnz/col, row scales 10^U(-4,4) and
  column scales 10^U(-3,3).

All generators are vectorised numpy and deterministic in their seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

LE, EQ, GE = 0, 1, 2


@dataclass
class LP:
    """An LP in original row form: min/max obj.x  s.t.  row_i(x) sense_i rhs_i, lb <= x <= ub."""

    m: int
    n: int
    rowptr: np.ndarray          # int32 [m+1]
    colidx: np.ndarray          # int32 [nnz], strictly ascending within a row
    vals: np.ndarray            # float64 [nnz]
    sense: np.ndarray           # int32 [m]  (LE, EQ, GE)
    rhs: np.ndarray             # float64 [m]
    obj: np.ndarray             # float64 [n]
    lb: np.ndarray              # float64 [n]
    ub: np.ndarray              # float64 [n]
    maximize: bool = False
    name: str = "lp"
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def standard(self) -> "StdLP":
        """Standard form of src/first_order_solver.cpp:68-101 (no presolve): >= rows negated,
        = rows flagged, objective multiplied by the sense (max -> -obj)."""
        row_of = np.repeat(np.arange(self.m), np.diff(self.rowptr))
        mult = np.where(self.sense == GE, -1.0, 1.0)
        vals = self.vals * mult[row_of]
        b = self.rhs * mult
        c = -self.obj if self.maximize else self.obj.copy()
        return StdLP(self.m, self.n, self.rowptr.astype(np.int32), self.colidx.astype(np.int32),
                     vals.astype(np.float64), b.astype(np.float64), c.astype(np.float64),
                     self.lb.astype(np.float64), self.ub.astype(np.float64),
                     (self.sense == EQ).astype(np.uint8), name=self.name)


@dataclass
class StdLP:
    """min c.x  s.t.  (A x)_i <= b_i (is_eq=0) or = b_i (is_eq=1),  lb <= x <= ub."""

    m: int
    n: int
    rowptr: np.ndarray
    colidx: np.ndarray
    vals: np.ndarray
    b: np.ndarray
    c: np.ndarray
    lb: np.ndarray
    ub: np.ndarray
    is_eq: np.ndarray
    name: str = "std"

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def spmv(self, x: np.ndarray) -> np.ndarray:
        row_of = np.repeat(np.arange(self.m), np.diff(self.rowptr))
        return np.bincount(row_of, weights=self.vals * x[self.colidx], minlength=self.m)

    def spmv_t(self, y: np.ndarray) -> np.ndarray:
        row_of = np.repeat(np.arange(self.m), np.diff(self.rowptr))
        return np.bincount(self.colidx, weights=self.vals * y[row_of], minlength=self.n)


def _csr_from_columns(m: int, n: int, col_rows: np.ndarray, col_of: np.ndarray, vals: np.ndarray):
    """Build a row-sorted CSR (column indices ascending within a row) from COO entries,
    summing duplicates and dropping explicit zeros as CSRMatrix::from_coo does
    (src/sparse_matrix.cpp:59-111)."""
    key = col_rows.astype(np.int64) * n + col_of.astype(np.int64)
    uk, inv = np.unique(key, return_inverse=True)
    v = np.bincount(inv, weights=vals, minlength=uk.size)
    keep = v != 0.0
    uk, v = uk[keep], v[keep]
    r = (uk // n).astype(np.int64)
    c = (uk % n).astype(np.int32)
    rowptr = np.zeros(m + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(np.bincount(r, minlength=m))
    return rowptr.astype(np.int32), c, v


def _distinct_rows_per_column(rng: np.random.Generator, m: int, n: int, k: np.ndarray | int) -> tuple:
    """For every column j draw k_j distinct rows uniformly from [0, m). Returns (rows, cols)."""
    k = np.broadcast_to(np.asarray(k), (n,)).astype(np.int64)
    kmax = int(k.max())
    # Rejection-free: sample kmax+4 candidates per column, keep the first k_j distinct ones.
    cand = rng.integers(0, m, size=(n, kmax + 6))
    s = np.sort(cand, axis=1)
    dup = np.zeros_like(s, dtype=bool)
    dup[:, 1:] = s[:, 1:] == s[:, :-1]
    # Random order of the distinct candidates, so the choice is uniform.
    keys = rng.random(s.shape)
    keys[dup] = 2.0
    idx = np.argsort(keys, axis=1)
    s = np.take_along_axis(s, idx, axis=1)
    ok = np.take_along_axis(~dup, idx, axis=1)
    # columns whose candidate pool held fewer than k_j distinct rows (small m): draw those
    # columns again without replacement, one by one
    for j in np.nonzero(ok.sum(axis=1) < k)[0]:
        s[j, :k[j]] = np.sort(rng.choice(m, size=int(k[j]), replace=False))
    take = np.arange(kmax + 6)[None, :] < k[:, None]
    rows = s[take]
    cols = np.repeat(np.arange(n), k)
    return rows, cols


def _finish(rng, m, n, rows, cols, vals, x0, sense, slack_scale, lb, ub, obj, name, meta=None, maximize=False):
    rowptr, colidx, v = _csr_from_columns(m, n, rows, cols, vals)
    row_of = np.repeat(np.arange(m), np.diff(rowptr))
    ax0 = np.bincount(row_of, weights=v * x0[colidx], minlength=m)
    slack = rng.random(m) * slack_scale
    rhs = np.where(sense == LE, ax0 + slack, np.where(sense == GE, ax0 - slack, ax0))
    return LP(m, n, rowptr, colidx, v, sense.astype(np.int32), rhs, obj, lb, ub, maximize, name, meta or {})


def random_sparse(m: int = 300, n: int = 1000, nnz_per_col: int = 5, seed: int = 0, name: str | None = None) -> LP:
    """Random sparse LP: half the rows '=' (even rows), half '<='; values +-U(0.1,10);
    x0 ~ U(0,1); b = A x0 (+U(0,1) slack on <= rows); 0 <= x <= 10; c ~ U(-1,1)."""
    rng = np.random.default_rng(seed)
    rows, cols = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    vals = rng.uniform(0.1, 10.0, rows.size) * rng.choice([-1.0, 1.0], rows.size)
    x0 = rng.random(n)
    sense = np.where(np.arange(m) % 2 == 0, EQ, LE)
    lb = np.zeros(n)
    ub = np.full(n, 10.0)
    obj = rng.uniform(-1.0, 1.0, n)
    return _finish(rng, m, n, rows, cols, vals, x0, sense, 1.0, lb, ub, obj, name or f"random_sparse_{m}x{n}_s{seed}")


def block_angular(periods: int = 50, block_rows: int = 4000, block_cols: int = 20000, nnz_per_col: int = 8,
                  link_rows: int = 4000, seed: int = 1) -> LP:
    """Multi-period blending LP: `periods` independent blocks (rows cycle <=, >=, = as the
    reference's BenchmarkGenerator does) plus `link_rows` inventory-balance equalities
    inv_t - inv_{t-1} + flows_t = d_t that tie consecutive periods together.

    Linking row r belongs to item k = r % items and period t = r // items
    (items = link_rows // periods); inv_{k,t} is column k of block t, and three flow
    columns of block t enter with lognormal coefficients. Feasible by construction
    (b = A x0); d_t is the resulting rhs of each balance row."""
    rng = np.random.default_rng(seed)
    m = periods * block_rows + link_rows
    n = periods * block_cols
    # block entries
    rows_b, cols_b = _distinct_rows_per_column(rng, block_rows, n, nnz_per_col)
    blk = cols_b // block_cols
    rows_b = rows_b + blk * block_rows
    items = link_rows // periods
    # linking entries: each linking row (k, t) gets +1 on inv_{k,t}, -1 on inv_{k,t-1}, 3 flows
    lr = np.arange(link_rows)
    k = lr % items
    t = lr // items
    inv_col = t * block_cols + k
    prev_col = (t - 1) * block_cols + k
    flow_cols = t[:, None] * block_cols + items + rng.integers(0, block_cols - items, size=(link_rows, 3))
    link_r = [lr, lr[t > 0]]
    link_c = [inv_col, prev_col[t > 0]]
    link_v = [np.ones(link_rows), -np.ones(int((t > 0).sum()))]
    link_r.append(np.repeat(lr, 3))
    link_c.append(flow_cols.ravel())
    link_v.append(rng.lognormal(0.0, 1.0, 3 * link_rows) * rng.choice([-1.0, 1.0], 3 * link_rows))
    rows = np.concatenate([rows_b] + [periods * block_rows + r for r in link_r])
    cols = np.concatenate([cols_b] + link_c)
    vals = np.concatenate([rng.lognormal(0.0, 1.0, rows_b.size) * rng.choice([-1.0, 1.0], rows_b.size)] + link_v)
    ub = rng.uniform(1.0, 100.0, n)
    lb = np.zeros(n)
    x0 = rng.random(n) * ub
    sense = np.concatenate([np.arange(periods * block_rows) % 3, np.full(link_rows, EQ)])
    sense = np.where(sense == 0, LE, np.where(sense == 1, GE, EQ)).astype(np.int32)
    sense[periods * block_rows:] = EQ
    obj = rng.standard_normal(n)
    return _finish(rng, m, n, rows, cols, vals, x0, sense, 1.0, lb, ub, obj,
                   f"block_angular_{periods}x{block_rows}x{block_cols}",
                   {"periods": periods, "block_rows": block_rows, "block_cols": block_cols, "link_rows": link_rows})


def uneven_batch(count: int = 4096, m_lo: int = 50, m_hi: int = 2000, seed: int = 2) -> list:
    """`count` independent random sparse LPs of uneven size: m ~ logU(m_lo, m_hi),
    n = m * U(2, 5), 4-10 nnz per column, values +-U(0.1,10), x0 construction as random_sparse."""
    rng = np.random.default_rng(seed)
    ms = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), count)).astype(np.int64)
    ns = (ms * rng.uniform(2.0, 5.0, count)).astype(np.int64)
    seeds = rng.integers(0, 2**63 - 1, count)
    out = []
    for i in range(count):
        out.append(_uneven_one(int(ms[i]), int(ns[i]), int(seeds[i]), f"batch{i}"))
    return out


def _uneven_one(m: int, n: int, seed: int, name: str) -> LP:
    rng = np.random.default_rng(seed)
    k = rng.integers(4, 11, n)
    k = np.minimum(k, m)
    rows, cols = _distinct_rows_per_column(rng, m, n, k)
    vals = rng.uniform(0.1, 10.0, rows.size) * rng.choice([-1.0, 1.0], rows.size)
    x0 = rng.random(n)
    sense = np.where(np.arange(m) % 2 == 0, EQ, LE)
    return _finish(rng, m, n, rows, cols, vals, x0, sense, 1.0, np.zeros(n), np.full(n, 10.0),
                   rng.uniform(-1.0, 1.0, n), name)


def ill_conditioned(m: int = 1_000_000, n: int = 5_000_000, nnz_per_col: int = 10, seed: int = 4) -> LP:
    """Badly scaled LP: entries +-U(0.1,10) times row scale 10^U(-4,4) times column scale
    10^U(-3,3); box [0, 10^U(0,3)]; c ~ N(0,1); b = A x0 (rows cycle <=, >=, =)."""
    rng = np.random.default_rng(seed)
    rows, cols = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    rs = 10.0 ** rng.uniform(-4.0, 4.0, m)
    cs = 10.0 ** rng.uniform(-3.0, 3.0, n)
    vals = rng.uniform(0.1, 10.0, rows.size) * rng.choice([-1.0, 1.0], rows.size) * rs[rows] * cs[cols]
    ub = 10.0 ** rng.uniform(0.0, 3.0, n)
    x0 = rng.random(n) * ub
    sense = np.arange(m) % 3
    sense = np.where(sense == 0, LE, np.where(sense == 1, GE, EQ)).astype(np.int32)
    lp = _finish(rng, m, n, rows, cols, vals, x0, sense, 0.0, np.zeros(n), ub, rng.standard_normal(n),
                 f"ill_conditioned_{m}x{n}")
    # slack on inequality rows scaled by the row's own magnitude
    slack = rng.random(m) * rs
    lp.rhs = np.where(sense == LE, lp.rhs + slack, np.where(sense == GE, lp.rhs - slack, lp.rhs))
    return lp


class RefineryFamily:
    """Parametric refinery-planning LP family on one fixed sparse structure.

    Structure (seed-fixed, n=8000 columns, m=2000 rows, 6 nnz per column):
      * 1000 mass-balance rows (=, rhs 0): each process column consumes and produces
        streams, so x = 0 always satisfies them;
      * 500 crude/unit availability rows (<=, positive coefficients, rhs > 0);
      * 500 product demand rows (>=, rhs > 0), each with one dedicated "spot purchase"
        column (cost 50-100) so every demand level is reachable -> feasible for every
        parameter vector, and bounded by the box 0 <= x <= ub.
    Parameters p in R^256: p[0:128] price multipliers U(0.8,1.2) (one per group of
    process columns), p[128:192] availability rhs scales U(0.7,1.3), p[192:256] demand
    rhs scales U(0.7,1.3) (groups of rows)."""

    N_PARAM = 256

    def __init__(self, m: int = 2000, n: int = 8000, nnz_per_col: int = 6, seed: int = 3):
        rng = np.random.default_rng(seed)
        self.m, self.n = m, n
        n_bal, n_av = m // 2, m // 4
        n_dem = m - n_bal - n_av
        self.n_bal, self.n_av, self.n_dem = n_bal, n_av, n_dem
        n_proc = n - n_dem
        # process columns: 2 balance entries (one +, one -), 2 availability, 2 demand/balance
        rows, cols, vals = [], [], []
        pc = np.arange(n_proc)
        bal = _distinct_rows_per_column(rng, n_bal, n_proc, 3)[0].reshape(n_proc, 3)
        av = rng.integers(0, n_av, size=(n_proc, 2))
        av[:, 1] = (av[:, 0] + 1 + rng.integers(0, n_av - 1, n_proc)) % n_av
        dem = rng.integers(0, n_dem, n_proc)
        rows += [bal[:, 0], bal[:, 1], bal[:, 2], n_bal + av[:, 0], n_bal + av[:, 1], n_bal + n_av + dem]
        cols += [pc] * 6
        sgn = rng.choice([-1.0, 1.0], size=(n_proc, 3))
        vals += [sgn[:, 0] * rng.uniform(0.5, 2.0, n_proc), sgn[:, 1] * rng.uniform(0.5, 2.0, n_proc),
                 sgn[:, 2] * rng.uniform(0.5, 2.0, n_proc), rng.uniform(0.2, 3.0, n_proc),
                 rng.uniform(0.2, 3.0, n_proc), rng.uniform(0.5, 2.0, n_proc)]
        # spot purchase columns: one per demand row (+1), plus 5 balance-free filler entries
        sp = n_proc + np.arange(n_dem)
        rows.append(n_bal + n_av + np.arange(n_dem))
        cols.append(sp)
        vals.append(np.ones(n_dem))
        for _ in range(nnz_per_col - 1):
            rows.append(n_bal + rng.integers(0, n_av, n_dem))
            cols.append(sp)
            vals.append(rng.uniform(0.01, 0.05, n_dem))
        rows = np.concatenate(rows)
        cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        # duplicates (a spot column may hit the same availability row twice) are summed
        self.rowptr, self.colidx, self.vals = _csr_from_columns(m, n, rows, cols, vals)
        self.sense = np.concatenate([np.full(n_bal, EQ), np.full(n_av, LE), np.full(n_dem, GE)]).astype(np.int32)
        self.base_cost = np.concatenate([rng.uniform(-3.0, 2.0, n_proc), rng.uniform(50.0, 100.0, n_dem)])
        self.ub = np.concatenate([rng.uniform(5.0, 50.0, n_proc), np.full(n_dem, 1e3)])
        row_of = np.repeat(np.arange(m), np.diff(self.rowptr))
        self.base_av = np.bincount(row_of, weights=self.vals * (0.3 * self.ub)[self.colidx], minlength=m)[n_bal:n_bal + n_av]
        self.base_dem = rng.uniform(20.0, 60.0, n_dem)
        self.price_group = np.concatenate([pc % 128, np.full(n_dem, -1)])
        self.av_group = np.arange(n_av) % 64
        self.dem_group = np.arange(n_dem) % 64

    def sample_params(self, count: int, seed: int, spread: float = 1.0) -> np.ndarray:
        """Price multipliers U(0.8, 1.2), rhs scales U(0.7, 1.3); `spread` < 1 narrows
        both ranges around 1 (a family whose solution map is nearly linear)."""
        rng = np.random.default_rng(seed)
        p = np.empty((count, self.N_PARAM))
        p[:, :128] = rng.uniform(0.8, 1.2, (count, 128))
        p[:, 128:] = rng.uniform(0.7, 1.3, (count, 128))
        return 1.0 + spread * (p - 1.0)

    def costs(self, p: np.ndarray) -> np.ndarray:
        mult = np.where(self.price_group >= 0, p[..., np.maximum(self.price_group, 0)], 1.0)
        return self.base_cost * mult

    def rhs(self, p: np.ndarray) -> np.ndarray:
        out = np.zeros(p.shape[:-1] + (self.m,))
        out[..., self.n_bal:self.n_bal + self.n_av] = self.base_av * p[..., 128 + self.av_group]
        out[..., self.n_bal + self.n_av:] = self.base_dem * p[..., 192 + self.dem_group]
        return out

    def instance(self, p: np.ndarray, name: str = "refinery") -> LP:
        return LP(self.m, self.n, self.rowptr, self.colidx, self.vals, self.sense, self.rhs(p), self.costs(p),
                  np.zeros(self.n), self.ub.copy(), False, name)

    def standard_batch(self, P: np.ndarray):
        """(shared standard-form matrix as a StdLP of the first instance, B, C, LB, UB, IS_EQ)
        for parameter vectors P [count x 256]: >= rows negated as in LP.standard()."""
        P = np.atleast_2d(P)
        s0 = self.instance(P[0]).standard()
        mult = np.where(self.sense == GE, -1.0, 1.0)
        count = P.shape[0]
        return (s0, self.rhs(P) * mult, self.costs(P), np.zeros((count, self.n)), np.tile(self.ub, (count, 1)),
                np.tile(s0.is_eq, (count, 1)))


class RefineryPlanningFamily:
    """Parametric multi-site refinery planning LP on one fixed structure.

    m = 2000 rows, n = 8000 columns, 6 nonzeros per column on average (seed-fixed):

    * market (192 rows): 96 crude-grade availability rows (<=), each grade contracted
      to two neighbouring sites (site s buys grades 6s .. 6s+11 mod 96, and the
      contracted volumes stay below the sites' distillation capacity), and 96
      (product, region) demand rows (>=), each with an import column (cost 1.5x the
      base product price: demand is always coverable -> feasible for every
      parameter vector);
    * 16 sites of 113 rows / 494 columns each:
        - 12 crude tanks (=): purchases of the site's 12 grades feed them;
        - 2 crude distillation units (capacity <=), 3 cut-point modes per (crude,
          unit): a run draws from the tank and yields 8 cut streams;
        - 40 stream balances (=): 16 cuts and 24 intermediates;
        - 12 conversion units (capacity <=), 6 modes each: one feed stream into
          three product streams (yields summing to 0.95);
        - 8 product pools: volume balance (=) and 4 linear blending-quality specs
          (<=: sum over streams of (quality - spec) * volume <= 0);
        - 7 utility balances (<=, purchasable at a cost) charged by runs and modes;
        - blending columns (stream -> pool), sales columns (pool -> demand row of 6
          reachable regions, bounded), stream disposal to fuel;
    * every column is boxed (0 <= x <= ub): bounded.

    Parameters p in R^256, as a planning department's scenario generator draws
    them: p[0:64] crude price multipliers U(0.8, 1.2) (grade g -> p[g % 64]),
    p[64:128] product price multipliers U(0.8, 1.2) ((product, region) pair k ->
    p[64 + k % 64]), p[128:192] availability scales U(0.7, 1.3) (crude grade g ->
    p[128 + g % 48], unit capacities -> p[176 + j % 16]), p[192:256] demand scales
    U(0.7, 1.3) (pair k -> p[192 + k % 64])."""

    N_PARAM = 256
    SITES, GRADES, PRODUCTS, REGIONS = 16, 96, 8, 12
    SITE_ROWS, SITE_COLS = 113, 494

    def __init__(self, seed: int = 3):
        rng = np.random.default_rng(seed)
        S, G, P, R = self.SITES, self.GRADES, self.PRODUCTS, self.REGIONS
        K = P * R
        rows, cols, vals = [], [], []
        cost, ub = [], []
        # parameter hooks per column: kind 0 none, 1 crude price, 2 product price
        cpar_kind, cpar_idx = [], []
        base_price = np.array([100.0, 95.0, 98.0, 85.0, 60.0, 50.0, 75.0, 90.0])
        prod_price = base_price[:, None] * rng.uniform(0.95, 1.05, (P, R))  # [P, R]
        crude_price = rng.uniform(55.0, 75.0, G)
        self.n_rows_market = G + K
        m = self.n_rows_market + S * self.SITE_ROWS
        sense = np.empty(m, np.int32)
        rhs_base = np.zeros(m)
        # parameter hooks per row: kind 0 none, 1 availability, 2 capacity, 3 demand
        rpar_kind = np.zeros(m, np.int32)
        rpar_idx = np.zeros(m, np.int32)
        avail_row = np.arange(G)
        dem_row = G + np.arange(K)
        sense[avail_row] = LE
        rhs_base[avail_row] = rng.uniform(20.0, 45.0, G)
        rpar_kind[avail_row], rpar_idx[avail_row] = 1, np.arange(G) % 48
        sense[dem_row] = GE
        rhs_base[dem_row] = rng.uniform(20.0, 60.0, K)
        rpar_kind[dem_row], rpar_idx[dem_row] = 3, np.arange(K) % 64
        col = 0

        def add(rlist, vlist, c, u, kind=0, idx=0):
            nonlocal col
            rows.append(np.asarray(rlist, np.int64))
            vals.append(np.asarray(vlist, np.float64))
            cols.append(np.full(len(rlist), col, np.int64))
            cost.append(c)
            ub.append(u)
            cpar_kind.append(kind)
            cpar_idx.append(idx)
            col += 1

        for k in range(K):  # imports, one per demand row
            add([dem_row[k]], [1.0], 1.5 * base_price[k // R], 1e4)
        cap_counter = 0
        for s in range(S):
            r0 = self.n_rows_market + s * self.SITE_ROWS
            tank = r0 + np.arange(12)
            cdu = r0 + 12 + np.arange(2)
            stream = r0 + 14 + np.arange(40)
            unit = r0 + 54 + np.arange(12)
            pool = r0 + 66 + np.arange(P)
            qual = r0 + 74 + np.arange(P * 4).reshape(P, 4)
            util = r0 + 106 + np.arange(7)
            sense[tank] = EQ
            sense[stream] = EQ
            sense[pool] = EQ
            sense[cdu] = LE
            sense[unit] = LE
            sense[qual.ravel()] = LE
            sense[util] = LE
            rhs_base[cdu] = rng.uniform(250.0, 450.0, 2)
            rhs_base[unit] = rng.uniform(40.0, 120.0, 12)
            for r_ in list(cdu) + list(unit):
                rpar_kind[r_], rpar_idx[r_] = 2, cap_counter % 16
                cap_counter += 1
            grades = (s * (G // S) + np.arange(12)) % G  # each grade is contracted to two neighbouring sites
            regions = rng.choice(R, 6, replace=False)
            qs = rng.uniform(0.0, 1.0, (40, 4))  # stream qualities
            spec = rng.uniform(0.35, 0.65, (P, 4))  # product specs
            for t, g in enumerate(grades):  # purchases
                add([tank[t], avail_row[g]], [1.0, 1.0], crude_price[g], 1e4, 1, g % 64)
            for t, g in enumerate(grades):  # distillation runs: (crude, unit, cut-point mode) -> 8 cuts
                base_y = rng.dirichlet(np.full(8, 2.0))
                for u in range(2):
                    for mode in range(3):
                        y = base_y * rng.uniform(0.8, 1.2, 8)
                        y = 0.98 * y / y.sum()
                        uu = rng.choice(7, 2, replace=False)
                        add([tank[t], cdu[u]] + list(stream[u * 8 + np.arange(8)]) + list(util[uu]),
                            [-1.0, 1.0] + list(y) + list(rng.uniform(0.01, 0.05, 2)), rng.uniform(0.5, 1.5), 1e3)
            for j in range(12):  # conversion unit modes: feed -> three intermediates
                for mode in range(6):
                    feed = rng.integers(0, 40)
                    outs = 16 + rng.choice(24, 3, replace=False)
                    outs = outs[outs != feed][:3]
                    while len(outs) < 3:
                        extra = 16 + rng.integers(0, 24)
                        if extra != feed and extra not in outs:
                            outs = np.append(outs, extra)
                    y = rng.dirichlet(np.full(3, 2.0)) * 0.95
                    uu = rng.choice(7, 2, replace=False)
                    add([stream[feed], unit[j]] + list(stream[outs]) + list(util[uu]),
                        [-1.0, 1.0] + list(y) + list(rng.uniform(0.02, 0.1, 2)), rng.uniform(1.0, 5.0), 1e3)
            for p_ in range(P):  # sales: pool -> reachable regions (bounded), revenue net of transport
                for r_ in regions:
                    k = p_ * R + r_
                    add([pool[p_], dem_row[k]], [-1.0, 1.0], -prod_price[p_, r_] + rng.uniform(1.0, 5.0),
                        rng.uniform(80.0, 200.0), 2, k % 64)
            for q in range(40):  # disposal of streams to fuel
                add([stream[q]], [-1.0], -rng.uniform(20.0, 35.0), 1e3)
            for q in range(7):  # utility purchase
                add([util[q]], [-1.0], rng.uniform(5.0, 15.0), 1e3)
            # blending: the site's remaining columns are (stream -> pool) options
            n_blend = self.SITE_COLS - (12 + 72 + 72 + P * 6 + 40 + 7)
            pairs = np.array([(q, p_) for q in range(40) for p_ in range(P)])
            pick = pairs[np.sort(rng.choice(len(pairs), n_blend, replace=False))]
            for q, p_ in pick:
                add([stream[q], pool[p_]] + list(qual[p_]), [-1.0, 1.0] + list(qs[q] - spec[p_]), 0.0, 1e3)
        n = col
        rows = np.concatenate(rows)
        cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        self.m, self.n = m, n
        self.rowptr, self.colidx, self.vals = _csr_from_columns(m, n, rows, cols, vals)
        self.sense = sense
        self.rhs_base = rhs_base
        self.rpar_kind, self.rpar_idx = rpar_kind, rpar_idx
        self.base_cost = np.asarray(cost)
        self.cpar_kind = np.asarray(cpar_kind, np.int32)
        self.cpar_idx = np.asarray(cpar_idx, np.int32)
        self.ub = np.asarray(ub)
        self.lb = np.zeros(n)

    def sample_params(self, count: int, seed: int, spread: float = 1.0) -> np.ndarray:
        """Price multipliers U(0.8, 1.2), rhs scales U(0.7, 1.3); `spread` < 1 narrows
        both ranges around 1 (a family whose solution map is nearly linear)."""
        rng = np.random.default_rng(seed)
        p = np.empty((count, self.N_PARAM))
        p[:, :128] = rng.uniform(0.8, 1.2, (count, 128))
        p[:, 128:] = rng.uniform(0.7, 1.3, (count, 128))
        return 1.0 + spread * (p - 1.0)

    def costs(self, p: np.ndarray) -> np.ndarray:
        p = np.asarray(p)
        col = np.where(self.cpar_kind == 1, self.cpar_idx, np.where(self.cpar_kind == 2, 64 + self.cpar_idx, 0))
        mult = np.where(self.cpar_kind[None, :] > 0, p.reshape(-1, self.N_PARAM)[:, col], 1.0)
        return (self.base_cost * mult).reshape(p.shape[:-1] + (self.n,))

    def rhs(self, p: np.ndarray) -> np.ndarray:
        p = np.asarray(p)
        idx = np.select([self.rpar_kind == 1, self.rpar_kind == 2, self.rpar_kind == 3],
                        [128 + self.rpar_idx, 176 + self.rpar_idx, 192 + self.rpar_idx], 0)
        mult = np.where(self.rpar_kind[None, :] > 0, p.reshape(-1, self.N_PARAM)[:, idx], 1.0)
        return (self.rhs_base * mult).reshape(p.shape[:-1] + (self.m,))

    def instance(self, p: np.ndarray, name: str = "refinery_planning") -> LP:
        return LP(self.m, self.n, self.rowptr, self.colidx, self.vals, self.sense, self.rhs(p), self.costs(p),
                  self.lb.copy(), self.ub.copy(), False, name)

    def standard_batch(self, P: np.ndarray):
        """(shared standard-form matrix as a StdLP of the first instance, B, C, LB, UB, IS_EQ)
        for parameter vectors P [count x 256]: >= rows negated as in LP.standard()."""
        P = np.atleast_2d(P)
        s0 = self.instance(P[0]).standard()
        mult = np.where(self.sense == GE, -1.0, 1.0)
        count = P.shape[0]
        return (s0, self.rhs(P) * mult, self.costs(P), np.tile(self.lb, (count, 1)), np.tile(self.ub, (count, 1)),
                np.tile(s0.is_eq, (count, 1)))
