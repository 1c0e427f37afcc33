"""LP model in the reference's shape (include/markov_cero/model/model.hpp:53-70).

The reference stores CSC with ``std::size_t`` indices and typed bounds
(``BoundKind``); this mirror stores CSC with int32 indices (the engine's
device layout) and +-inf for infinite bounds.  ``validate`` restates
``SparseMatrixCSC::validate`` (src/model/model.cpp:41-66) and the numeric
part of ``Model::validate`` (src/model/model.cpp:120-165); names and variable
types are not needed on the PDLP path and are not stored.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from ._abi import MC_MEMORY_HOST, McLp


class ObjectiveSense(enum.IntEnum):
    minimize = 0
    maximize = 1


@dataclass
class Model:
    num_rows: int
    num_cols: int
    col_start: np.ndarray          # int32 [n+1]
    row_index: np.ndarray          # int32 [nnz]
    value: np.ndarray              # float64 [nnz]
    objective: np.ndarray          # float64 [n]
    var_lower: np.ndarray          # float64 [n], -inf = unbounded
    var_upper: np.ndarray          # float64 [n], +inf = unbounded
    row_lower: np.ndarray          # float64 [m]
    row_upper: np.ndarray          # float64 [m]
    objective_offset: float = 0.0
    objective_sense: ObjectiveSense = ObjectiveSense.minimize
    name: str = ""
    info: dict = field(default_factory=dict)   # generator metadata (x*, y*, optimum)

    @property
    def nnz(self) -> int:
        return int(self.col_start[-1]) if len(self.col_start) else 0

    def __post_init__(self) -> None:
        self.col_start = np.ascontiguousarray(self.col_start, dtype=np.int32)
        self.row_index = np.ascontiguousarray(self.row_index, dtype=np.int32)
        for name in ("value", "objective", "var_lower", "var_upper", "row_lower", "row_upper"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.float64))

    def validate(self) -> None:
        """Raise ValueError like the reference raises std::invalid_argument."""
        m, n = self.num_rows, self.num_cols
        cs, ri, v = self.col_start, self.row_index, self.value
        if len(cs) != n + 1:
            raise ValueError("CSC column_start size mismatch")
        if len(cs) == 0 or cs[0] != 0:
            raise ValueError("CSC must start at zero")
        if len(ri) != len(v):
            raise ValueError("CSC index/value size mismatch")
        if cs[-1] != len(v):
            raise ValueError("CSC terminal pointer mismatch")
        if np.any(np.diff(cs.astype(np.int64)) < 0):
            raise ValueError("CSC pointers must be monotone")
        if len(ri) and (ri.min() < 0 or ri.max() >= m):
            raise ValueError("CSC row index out of range")
        if len(ri) > 1:
            d = np.diff(ri.astype(np.int64))
            first = np.zeros(len(ri), dtype=bool)
            first[cs[:-1][cs[:-1] < len(ri)]] = True
            if np.any((d <= 0) & ~first[1:]):
                raise ValueError("CSC rows must be strictly increasing per column")
        if not np.all(np.isfinite(v)) or np.any(v == 0.0):
            raise ValueError("CSC values must be finite and nonzero")
        if not np.isfinite(self.objective_offset):
            raise ValueError("objective offset must be finite")
        if len(self.objective) != n or len(self.var_lower) != n or len(self.var_upper) != n:
            raise ValueError("variable metadata dimension mismatch")
        if len(self.row_lower) != m or len(self.row_upper) != m:
            raise ValueError("row metadata dimension mismatch")
        if not np.all(np.isfinite(self.objective)):
            raise ValueError("objective coefficient must be finite")
        if np.any(np.isnan(self.var_lower)) or np.any(np.isnan(self.var_upper)):
            raise ValueError("variable bound must be finite")
        if np.any(self.var_lower == np.inf) or np.any(self.var_upper == -np.inf):
            raise ValueError("invalid variable infinity direction")
        if np.any(self.var_lower > self.var_upper):
            raise ValueError("inconsistent variable bounds")
        if np.any(np.isnan(self.row_lower)) or np.any(np.isnan(self.row_upper)):
            raise ValueError("row bound must be finite")
        if np.any(self.row_lower == np.inf) or np.any(self.row_upper == -np.inf):
            raise ValueError("invalid row infinity direction")
        if np.any(self.row_lower > self.row_upper):
            raise ValueError("inconsistent row bounds")

    def to_struct(self) -> McLp:
        """Host-memory mc_lp view (the arrays must outlive the struct)."""
        s = McLp()
        s.num_rows = self.num_rows
        s.num_cols = self.num_cols
        s.nnz = self.nnz
        s.col_start = self.col_start.ctypes.data
        s.row_index = self.row_index.ctypes.data
        s.value = self.value.ctypes.data
        s.objective = self.objective.ctypes.data
        s.var_lower = self.var_lower.ctypes.data
        s.var_upper = self.var_upper.ctypes.data
        s.row_lower = self.row_lower.ctypes.data
        s.row_upper = self.row_upper.ctypes.data
        s.objective_offset = float(self.objective_offset)
        s.objective_sense = int(self.objective_sense)
        s.memory = MC_MEMORY_HOST
        return s

    def copy(self) -> "Model":
        return Model(self.num_rows, self.num_cols, self.col_start.copy(), self.row_index.copy(),
                     self.value.copy(), self.objective.copy(), self.var_lower.copy(),
                     self.var_upper.copy(), self.row_lower.copy(), self.row_upper.copy(),
                     self.objective_offset, self.objective_sense, self.name, dict(self.info))


def from_triplets(m: int, n: int, rows, cols, vals, **kw) -> Model:
    """Build a Model like SparseMatrixBuilder (src/model/model.cpp:88-118):
    duplicates summed, zeros dropped, columns sorted by row."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    agg: dict[tuple[int, int], float] = {}
    for r, c, v in zip(rows.tolist(), cols.tolist(), vals.tolist()):
        agg[(c, r)] = agg.get((c, r), 0.0) + v
    keys = sorted(k for k, v in agg.items() if v != 0.0)
    col_start = np.zeros(n + 1, dtype=np.int32)
    for c, _ in keys:
        col_start[c + 1] += 1
    col_start = np.cumsum(col_start).astype(np.int32)
    row_index = np.array([r for _, r in keys], dtype=np.int32)
    value = np.array([agg[k] for k in keys], dtype=np.float64)
    return Model(m, n, col_start, row_index, value, **kw)


def csc_to_dense(model: Model) -> np.ndarray:
    A = np.zeros((model.num_rows, model.num_cols))
    for j in range(model.num_cols):
        for p in range(model.col_start[j], model.col_start[j + 1]):
            A[model.row_index[p], j] += model.value[p]
    return A


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)
