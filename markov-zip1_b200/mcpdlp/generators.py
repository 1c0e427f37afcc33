"""Seeded synthetic LP workloads (thin wrappers over gen/lpgen.c).

Families, sizes and distributions follow the engine's workloads:
  * ``random_lp``      -- equality-row LP with analytic optimum c.x* = b.y*
                          (k nonzeros per column, N(0,1) values, 0 <= x <= 10)
  * ``random_lp(..., family="precision")`` -- |a| log-uniform on [1e-3, 1e3]
                          with random sign; 20% of columns boxed by U(1,100)
  * ``transport``      -- transportation LP (supply <=, demand =, x >= 0)
  * ``tighten_bounds`` -- branch-and-bound style node variants of a base LP
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .model import Model, ObjectiveSense

FAMILIES = {"standard": 0, "precision": 1}

# Shapes of the named workloads.
CONFIG0 = dict(m=1000, n=3000, k=6)               # small LP with known optimum
CONFIG1 = dict(m=2_000_000, n=5_000_000, k=8)     # 40M nonzeros, FP64
CONFIG2 = dict(m=1_000_000, n=3_000_000, k=10, family="precision")  # 30M nonzeros


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def random_lp(seed: int, m: int, n: int, k: int, family: str = "standard") -> Model:
    lib = _lib.lpgen()
    nnz = n * k
    col_start = np.empty(n + 1, np.int32)
    row_index = np.empty(nnz, np.int32)
    value = np.empty(nnz, np.float64)
    objective = np.empty(n, np.float64)
    var_lower = np.empty(n, np.float64)
    var_upper = np.empty(n, np.float64)
    row_lower = np.empty(m, np.float64)
    row_upper = np.empty(m, np.float64)
    x_star = np.empty(n, np.float64)
    y_star = np.empty(m, np.float64)
    opt = np.empty(2, np.float64)
    rc = lib.lpgen_random_lp(seed, m, n, k, FAMILIES[family], _p(col_start), _p(row_index),
                             _p(value), _p(objective), _p(var_lower), _p(var_upper),
                             _p(row_lower), _p(row_upper), _p(x_star), _p(y_star), _p(opt))
    if rc != 0:
        raise ValueError(f"lpgen_random_lp rejected m={m} n={n} k={k} ({rc})")
    return Model(m, n, col_start, row_index, value, objective, var_lower, var_upper,
                 row_lower, row_upper, 0.0, ObjectiveSense.minimize,
                 name=f"random-{family}-s{seed}-{m}x{n}k{k}",
                 info=dict(x_star=x_star, y_star=y_star, optimum=float(opt[0]),
                           dual_optimum=float(opt[1]), seed=seed, family=family))


def transport(seed: int, S: int | None = None, D: int | None = None) -> Model:
    """Transportation LP; S and D default to U[50,500] drawn from the seed."""
    lib = _lib.lpgen()
    if S is None:
        S = int(lib.lpgen_uniform_int(seed, 0, 50, 500))
    if D is None:
        D = int(lib.lpgen_uniform_int(seed, 1, 50, 500))
    m, n = S + D, S * D
    col_start = np.empty(n + 1, np.int32)
    row_index = np.empty(2 * n, np.int32)
    value = np.empty(2 * n, np.float64)
    objective = np.empty(n, np.float64)
    var_lower = np.empty(n, np.float64)
    var_upper = np.empty(n, np.float64)
    row_lower = np.empty(m, np.float64)
    row_upper = np.empty(m, np.float64)
    sup = np.empty(2 * S, np.float64)
    dem = np.empty(2 * D, np.float64)
    rc = lib.lpgen_transport(seed, S, D, _p(col_start), _p(row_index), _p(value),
                             _p(objective), _p(var_lower), _p(var_upper), _p(row_lower),
                             _p(row_upper), _p(sup), _p(dem))
    if rc != 0:
        raise ValueError(f"lpgen_transport rejected S={S} D={D} ({rc})")
    return Model(m, n, col_start, row_index, value, objective, var_lower, var_upper,
                 row_lower, row_upper, 0.0, ObjectiveSense.minimize,
                 name=f"transport-s{seed}-{S}x{D}",
                 info=dict(S=S, D=D, supply_xy=sup.reshape(S, 2), demand_xy=dem.reshape(D, 2),
                           seed=seed))


def tighten_bounds(base: Model, seed: int) -> tuple[Model, np.ndarray]:
    """A node variant of ``base``: 1-10 bounds tightened around x*."""
    lib = _lib.lpgen()
    x_star = base.info["x_star"]
    lo = base.var_lower.copy()
    hi = base.var_upper.copy()
    cols = np.zeros(10, np.int32)
    cnt = lib.lpgen_tighten_bounds(seed, base.num_cols, _p(x_star), _p(lo), _p(hi), _p(cols))
    if cnt < 0:
        raise ValueError("lpgen_tighten_bounds failed")
    v = base.copy()
    v.var_lower, v.var_upper = lo, hi
    v.name = f"{base.name}-node{seed}"
    return v, cols[:cnt].copy()


def batch_part1_shapes(seed: int, count: int = 256, m_range=(100, 20000)) -> list:
    """(m, n, k) of the uneven batch: m ~ U[m_range], n ~ U[2m, 4m], k ~ U{4..12}."""
    lib = _lib.lpgen()
    out = []
    for b in range(count):
        m = int(lib.lpgen_uniform_int(seed, 3 * b, m_range[0], m_range[1]))
        n = int(lib.lpgen_uniform_int(seed, 3 * b + 1, 2 * m, 4 * m))
        k = int(lib.lpgen_uniform_int(seed, 3 * b + 2, 4, 12))
        out.append((m, n, k))
    return out


def batch_part1(seed: int, count: int = 256, m_range=(100, 20000), only=None) -> list:
    """Uneven batch: `count` LPs of the standard family with shapes from
    batch_part1_shapes (each from its own seed); `only` selects indices."""
    shapes = batch_part1_shapes(seed, count, m_range)
    idx = range(count) if only is None else only
    return [random_lp(seed * 100003 + b, *shapes[b]) for b in idx]


def batch_part2(seed: int, variants: int = 512, m: int = 5000, n: int = 15000, k: int = 8, only=None):
    """One base LP and `variants` node variants (1-10 bounds tightened to
    floor/ceil of x* -+ U(0,1)); returns (base, [variants], [tightened cols]);
    `only` selects variant indices."""
    base = random_lp(seed, m, n, k)
    vs, cols = [], []
    for v in (range(variants) if only is None else only):
        mv, cv = tighten_bounds(base, seed * 7919 + v)
        vs.append(mv)
        cols.append(cv)
    return base, vs, cols


def uniform_int(seed: int, index: int, lo: int, hi: int) -> int:
    return int(_lib.lpgen().lpgen_uniform_int(seed, index, lo, hi))


def presolve_lp(seed: int, m: int, n: int, k: int = 3, singletons: float = 0.05, chains: int = 4,
                chain_len: int = 6, empty_rows: float = 0.01, empty_cols: float = 0.01, tiny: float = 0.01,
                kind: str = "feasible"):
    """A canonical model (min c.x, A x = rhs, x >= 0) shaped to exercise
    presolve: about k entries per column; a `singletons` share of rows cut to
    one entry; `chains` staircases of `chain_len` rows (row t holds the
    columns of steps t-1 and t) in increasing row order, so that each
    singleton makes the next row one, and as many in decreasing row order
    (one step per pass); empty rows and columns; a `tiny` share of entries at
    1e-13 (below the default pivot tolerance).  rhs = A x* for x* >= 0, so the
    singletons fix non-negative values.  kind = "infeasible_row" adds an empty
    row with rhs 1; "infeasible_singleton" a singleton row fixing -1;
    "unbounded" an empty column with cost -1.  Returns a CanonicalModel."""
    from .presolve import CanonicalModel
    rng = np.random.default_rng(seed)
    rows_of = [set(rng.choice(m, size=min(k, m), replace=False).tolist()) for _ in range(n)]
    # empty columns
    for j in rng.choice(n, size=int(empty_cols * n), replace=False):
        rows_of[j] = set()
    # staircases: forward (increasing rows) and backward (decreasing rows)
    used_cols = set()
    for c in range(2 * chains):
        rows = np.sort(rng.choice(m, size=chain_len, replace=False))
        if c % 2:
            rows = rows[::-1]
        cols = [j for j in rng.permutation(n)[:4 * chain_len] if j not in used_cols][:chain_len]
        if len(cols) < chain_len:
            continue
        used_cols.update(cols)
        for j in cols:
            rows_of[j].difference_update(rows.tolist())
        for t, r in enumerate(rows):
            # row r keeps only cols[t] (and cols[t-1]) among all columns
            for j in range(n):
                if r in rows_of[j] and j != cols[t] and (t == 0 or j != cols[t - 1]):
                    rows_of[j].discard(r)
            rows_of[cols[t]].add(int(r))
            if t > 0:
                rows_of[cols[t - 1]].add(int(r))
    # singleton rows: keep one random entry of the row
    entries = {}
    for j in range(n):
        for r in rows_of[j]:
            entries.setdefault(r, []).append(j)
    for r in rng.choice(m, size=int(singletons * m), replace=False):
        cols = entries.get(int(r), [])
        if len(cols) > 1:
            keep = cols[rng.integers(len(cols))]
            for j in cols:
                if j != keep:
                    rows_of[j].discard(int(r))
    # empty rows
    for r in rng.choice(m, size=int(empty_rows * m), replace=False):
        for j in range(n):
            rows_of[j].discard(int(r))
    col_start = [0]
    row_index, value = [], []
    for j in range(n):
        for r in sorted(rows_of[j]):
            v = rng.normal()
            if v == 0.0:
                v = 1.0
            if rng.random() < tiny:
                v = 1e-13 * (1 if v > 0 else -1)
            row_index.append(r)
            value.append(v)
        col_start.append(len(row_index))
    col_start = np.array(col_start, np.int32)
    row_index = np.array(row_index, np.int32)
    value = np.array(value)
    x = np.where(rng.random(n) < 0.3, 0.0, rng.uniform(0.5, 3.0, n))
    rhs = np.zeros(m)
    for j in range(n):
        for p in range(col_start[j], col_start[j + 1]):
            rhs[row_index[p]] += value[p] * x[j]
    obj = np.abs(rng.normal(size=n)) + 0.1
    if kind == "infeasible_row":
        r = int(rng.integers(m))
        keep = value != 0
        for j in range(n):
            for p in range(col_start[j], col_start[j + 1]):
                if row_index[p] == r:
                    keep[p] = False
        col_start = np.concatenate([[0], np.cumsum([keep[col_start[j]:col_start[j + 1]].sum()
                                                    for j in range(n)])]).astype(np.int32)
        row_index, value = row_index[keep], value[keep]
        rhs[r] = 1.0
    elif kind == "infeasible_singleton":
        # a new row with a single entry whose value forces x_j = -1
        j = int(rng.integers(n))
        m += 1
        rhs = np.append(rhs, -abs(value[col_start[j]]) if col_start[j + 1] > col_start[j] else -1.0)
        ins = col_start[j + 1]
        row_index = np.insert(row_index, ins, m - 1)
        value = np.insert(value, ins, 1.0)
        col_start[j + 1:] += 1
        rhs[-1] = -1.0
    elif kind == "unbounded":
        j = int(rng.integers(n))
        keep = np.ones(len(value), bool)
        keep[col_start[j]:col_start[j + 1]] = False
        col_start = np.concatenate([[0], np.cumsum([keep[col_start[q]:col_start[q + 1]].sum()
                                                    for q in range(n)])]).astype(np.int32)
        row_index, value = row_index[keep], value[keep]
        obj[j] = -1.0
    return CanonicalModel(m, n, col_start, row_index, value, rhs, obj, float(rng.normal()))


def presolve_workload(seed: int, m: int, n: int, k: int = 4, singletons: float = 0.05, chains: int = 64,
                      chain_len: int = 32, empty_rows: float = 0.01, empty_cols: float = 0.01,
                      tiny: float = 0.001):
    """A large canonical model for timing presolve, built with numpy only
    (presolve_lp's shape at scale): about k entries per column, a
    `singletons` share of rows cut to one entry, `chains` staircases of
    `chain_len` rows (half in increasing row order: one pass each; half
    decreasing: one step per pass), empty rows and columns, a `tiny` share of
    entries at 1e-13.  rhs = A x* for x* >= 0.  Returns a CanonicalModel."""
    from .presolve import CanonicalModel
    rng = np.random.default_rng(seed)
    cols = np.repeat(np.arange(n, dtype=np.int64), k)
    rows = rng.integers(0, m, size=n * k, dtype=np.int64)
    key = np.unique(cols * m + rows)  # distinct (column, row) pairs, column-major
    cols, rows = key // m, key % m
    drop = np.zeros(len(rows), bool)
    drop |= np.isin(rows, rng.choice(m, size=int(empty_rows * m), replace=False))
    drop |= np.isin(cols, rng.choice(n, size=int(empty_cols * n), replace=False))
    # staircases on fresh rows and columns
    c_rows = rng.choice(m, size=chains * chain_len, replace=False).reshape(chains, chain_len)
    c_rows.sort(axis=1)
    c_rows[1::2] = c_rows[1::2, ::-1]
    c_cols = rng.choice(n, size=chains * chain_len, replace=False).reshape(chains, chain_len)
    drop |= np.isin(rows, c_rows.ravel()) | np.isin(cols, c_cols.ravel())
    # singleton rows: one entry kept (the one with the smallest random key)
    s_rows = rng.choice(m, size=int(singletons * m), replace=False)
    in_s = np.isin(rows, s_rows) & ~drop
    idx = np.nonzero(in_s)[0]
    order = idx[np.lexsort((rng.random(len(idx)), rows[idx]))]
    first = np.ones(len(order), bool)
    first[1:] = rows[order[1:]] != rows[order[:-1]]
    drop[order[~first]] = True
    rows, cols = rows[~drop], cols[~drop]
    add_r = np.concatenate([c_rows.ravel(), c_rows[:, 1:].ravel()])
    add_c = np.concatenate([c_cols.ravel(), c_cols[:, :-1].ravel()])
    key = np.unique(np.concatenate([cols * m + rows, add_c * m + add_r]))
    cols, rows = key // m, key % m
    value = rng.normal(size=len(rows))
    value[value == 0.0] = 1.0
    t = rng.random(len(rows)) < tiny
    value[t] = np.copysign(1e-13, value[t])
    col_start = np.zeros(n + 1, np.int64)
    np.add.at(col_start, cols + 1, 1)
    col_start = np.cumsum(col_start).astype(np.int32)
    x = np.where(rng.random(n) < 0.3, 0.0, rng.uniform(0.5, 3.0, n))
    rhs = np.bincount(rows, weights=value * x[cols], minlength=m).astype(np.float64)
    obj = np.abs(rng.normal(size=n)) + 0.1
    return CanonicalModel(m, n, col_start, rows.astype(np.int32), value, rhs, obj, float(rng.normal()))
