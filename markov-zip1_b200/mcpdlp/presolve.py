"""Presolve of a canonical model on the GPU (mc_presolve_run / mc_postsolve).

Mirrors ``markov_cero::presolve`` (include/markov_cero/presolve/presolve.hpp,
presolve_stack.hpp; src/presolve/presolve.cpp:20-317)::

    res = presolve(model, PresolveOptions(), ctx=ctx)   # PresolveResult
    res.status, res.model, res.stack, res.statistics, res.message
    out = postsolve(res.stack, reduced_solution, model)  # primal, dual, objective

``model`` is a :class:`CanonicalModel` (SparseCanonicalModel: min c.x + offset,
A x = rhs, x >= 0, CSC).  The reduced model, the record stack and the maps are
bit-identical to the reference's; the reduction runs on the device, and so
does postsolve (its long double sums are double-double there).  A model the
reference's ``validate()`` rejects raises ``ValueError``.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import Context, _abi, _lib, _raise


class SolveStatus(enum.IntEnum):
    """lp::reference::SolveStatus values that presolve returns."""
    optimal = 0
    infeasible = 1
    unbounded = 2


@dataclass
class CanonicalModel:
    """SparseCanonicalModel (sparse_canonical_model.hpp:12-19) without its
    canonicalisation record, which presolve does not use."""
    num_rows: int
    num_cols: int
    col_start: np.ndarray
    row_index: np.ndarray
    value: np.ndarray
    rhs: np.ndarray
    objective: np.ndarray
    objective_offset: float = 0.0

    def __post_init__(self):
        self.col_start = np.ascontiguousarray(self.col_start, dtype=np.int32)
        self.row_index = np.ascontiguousarray(self.row_index, dtype=np.int32)
        self.value = np.ascontiguousarray(self.value, dtype=np.float64)
        self.rhs = np.ascontiguousarray(self.rhs, dtype=np.float64)
        self.objective = np.ascontiguousarray(self.objective, dtype=np.float64)

    @property
    def nnz(self) -> int:
        return int(len(self.value))

    def to_struct(self) -> _abi.McCanonicalLp:
        s = _abi.McCanonicalLp()
        s.num_rows, s.num_cols, s.nnz = self.num_rows, self.num_cols, self.nnz
        s.col_start = self.col_start.ctypes.data
        s.row_index = self.row_index.ctypes.data if self.nnz else None
        s.value = self.value.ctypes.data if self.nnz else None
        s.rhs = self.rhs.ctypes.data if self.num_rows else None
        s.objective = self.objective.ctypes.data if self.num_cols else None
        s.objective_offset = float(self.objective_offset)
        return s

    def dense(self) -> np.ndarray:
        a = np.zeros((self.num_rows, self.num_cols))
        for j in range(self.num_cols):
            for p in range(self.col_start[j], self.col_start[j + 1]):
                a[self.row_index[p], j] = self.value[p]
        return a


@dataclass
class PresolveOptions:
    """PresolveOptions (presolve.hpp:12-17)."""
    max_passes: int = 5
    feasibility_tolerance: float = 1e-9
    dual_tolerance: float = 1e-9
    pivot_tolerance: float = 1e-12

    def to_struct(self) -> _abi.McPresolveOptions:
        return _abi.McPresolveOptions(self.max_passes, self.feasibility_tolerance, self.dual_tolerance,
                                      self.pivot_tolerance)


@dataclass
class PresolveStatistics:
    """PresolveStatistics (presolve.hpp:19-29)."""
    passes_executed: int = 0
    empty_rows_removed: int = 0
    empty_cols_removed: int = 0
    fixed_vars_removed: int = 0
    row_singletons_removed: int = 0
    original_rows: int = 0
    original_cols: int = 0
    presolved_rows: int = 0
    presolved_cols: int = 0


# the ReductionRecord alternatives (presolve_stack.hpp:9-39)
@dataclass
class EmptyRowRecord:
    original_row_index: int
    rhs_value: float


@dataclass
class EmptyColumnRecord:
    original_col_index: int
    objective_coeff: float
    fixed_value: float


@dataclass
class FixedVariableRecord:
    original_col_index: int
    fixed_value: float
    objective_coeff: float
    row_indices: list
    coefficients: list


@dataclass
class RowSingletonRecord:
    original_row_index: int
    variable_index: int
    coefficient: float
    rhs_value: float


class _Handle:
    """Owns one mc_presolve (device memory), freed with the last reference."""

    def __init__(self, lib, ptr: C.c_void_p, device: int, rows: int, cols: int):
        self._lib, self.ptr, self.device = lib, ptr, device
        self.rows, self.cols = rows, cols  # of the model presolve ran on

    def __del__(self):
        try:
            if self.ptr:
                self._lib.mc_presolve_free(self.ptr)
                self.ptr = C.c_void_p()
        except Exception:
            pass


@dataclass
class PresolveStack:
    """PresolveStack (presolve_stack.hpp:41-72) as flat arrays, oldest record
    first: kind (mc_record_kind), index, variable, value, value2 and the
    fixed-variable records' incident rows (incident_start into incident_row
    and incident_coefficient)."""
    kind: np.ndarray
    index: np.ndarray
    variable: np.ndarray
    value: np.ndarray
    value2: np.ndarray
    incident_start: np.ndarray
    incident_row: np.ndarray
    incident_coefficient: np.ndarray
    presolved_to_original_rows: np.ndarray
    presolved_to_original_cols: np.ndarray
    handle: Optional[_Handle] = field(default=None, repr=False, compare=False)

    def size(self) -> int:
        return int(len(self.kind))

    def records(self) -> list:
        out = []
        for t, k in enumerate(self.kind.tolist()):
            if k == _abi.MC_RECORD_EMPTY_ROW:
                out.append(EmptyRowRecord(int(self.index[t]), float(self.value[t])))
            elif k == _abi.MC_RECORD_EMPTY_COLUMN:
                out.append(EmptyColumnRecord(int(self.index[t]), float(self.value[t]), float(self.value2[t])))
            elif k == _abi.MC_RECORD_FIXED_VARIABLE:
                a, b = int(self.incident_start[t]), int(self.incident_start[t + 1])
                out.append(FixedVariableRecord(int(self.index[t]), float(self.value[t]), float(self.value2[t]),
                                               self.incident_row[a:b].tolist(),
                                               self.incident_coefficient[a:b].tolist()))
            else:
                out.append(RowSingletonRecord(int(self.index[t]), int(self.variable[t]), float(self.value[t]),
                                              float(self.value2[t])))
        return out


@dataclass
class PresolveResult:
    """PresolveResult (presolve.hpp:31-37); extra: device timing and rounds."""
    status: SolveStatus
    model: CanonicalModel
    stack: PresolveStack
    statistics: PresolveStatistics
    message: str
    extra: dict = field(default_factory=dict)


@dataclass
class PostsolveResult:
    primal: np.ndarray
    dual: np.ndarray
    objective: float


def _info_to_result(info: _abi.McPresolveInfo) -> tuple:
    st = PresolveStatistics(*(int(getattr(info, f)) for f in (
        "passes_executed", "empty_rows_removed", "empty_cols_removed", "fixed_vars_removed",
        "row_singletons_removed", "original_rows", "original_cols", "presolved_rows", "presolved_cols")))
    return SolveStatus(info.status), st, info.message.decode()


def read_result(lib, ptr, info: _abi.McPresolveInfo, handle: Optional[_Handle]) -> PresolveResult:
    """Copies a presolve result out of the engine (arrays as numpy)."""
    status, st, msg = _info_to_result(info)
    nm, nn, nz = int(info.presolved_rows), int(info.presolved_cols), int(info.presolved_nnz)
    nr, ni = int(info.records), int(info.incident_entries)
    cs = np.zeros(nn + 1, np.int32)
    ri = np.zeros(nz, np.int32)
    v = np.zeros(nz)
    rhs = np.zeros(nm)
    obj = np.zeros(nn)
    p = lambda a: a.ctypes.data if a.size else None  # noqa: E731
    _raise(lib.mc_presolve_get_model(ptr, p(cs), p(ri), p(v), p(rhs), p(obj)))
    rmap = np.zeros(nm, np.int64)
    cmap = np.zeros(nn, np.int64)
    _raise(lib.mc_presolve_get_maps(ptr, p(rmap), p(cmap)))
    kind = np.zeros(nr, np.int32)
    index = np.zeros(nr, np.int64)
    var = np.zeros(nr, np.int64)
    val = np.zeros(nr)
    val2 = np.zeros(nr)
    ist = np.zeros(nr + 1, np.int64)
    irow = np.zeros(ni, np.int64)
    icoef = np.zeros(ni)
    _raise(lib.mc_presolve_get_records(ptr, p(kind), p(index), p(var), p(val), p(val2), p(ist), p(irow), p(icoef)))
    model = CanonicalModel(nm, nn, cs, ri, v, rhs, obj, float(info.objective_offset))
    stack = PresolveStack(kind, index, var, val, val2, ist, irow, icoef, rmap, cmap, handle)
    extra = dict(presolve_ms=float(info.presolve_ms), scan_rounds=int(info.scan_rounds),
                 presolved_nnz=nz, incident_entries=ni)
    return PresolveResult(status, model, stack, st, msg, extra)


def presolve(model: CanonicalModel, options: Optional[PresolveOptions] = None,
             ctx: Optional[Context] = None) -> PresolveResult:
    """presolve() (presolve.cpp:20) on the context's device."""
    ctx = ctx or Context(0)
    options = options or PresolveOptions()
    lib = _lib.engine()
    s = model.to_struct()
    o = options.to_struct()
    ptr = C.c_void_p()
    _raise(lib.mc_presolve_run(ctx.handle, C.byref(s), C.byref(o), C.byref(ptr)))
    handle = _Handle(lib, ptr, ctx.device, model.num_rows, model.num_cols)
    info = _abi.McPresolveInfo()
    _raise(lib.mc_presolve_get_info(ptr, C.byref(info)))
    res = read_result(lib, ptr, info, handle)
    res.extra["context"] = ctx
    return res


def postsolve(stack: PresolveStack, reduced_solution, original_model: CanonicalModel,
              tolerance: float = 1e-8, ctx: Optional[Context] = None) -> PostsolveResult:
    """postsolve() (presolve.cpp:219) on the device.  ``reduced_solution`` has
    ``primal`` and ``dual`` (a shorter array leaves the missing entries 0, as
    in the reference); ``original_model`` must be the model presolve ran on
    (the device keeps its own copy of it).  ``tolerance`` is unused, as in
    the reference."""
    if stack.handle is None or not stack.handle.ptr:
        raise ValueError("this stack holds no device presolve result")
    if (original_model.num_rows, original_model.num_cols) != (stack.handle.rows, stack.handle.cols):
        raise ValueError("original_model is not the model this stack was presolved from")
    ctx = ctx or Context(stack.handle.device)
    lib = _lib.engine()
    rx = np.ascontiguousarray(getattr(reduced_solution, "primal"), dtype=np.float64)
    ry = np.ascontiguousarray(getattr(reduced_solution, "dual"), dtype=np.float64)
    x = np.zeros(original_model.num_cols)
    y = np.zeros(original_model.num_rows)
    obj = C.c_double()
    p = lambda a: a.ctypes.data if a.size else None  # noqa: E731
    _raise(lib.mc_postsolve(ctx.handle, stack.handle.ptr, p(rx), len(rx), p(ry), len(ry), p(x), p(y),
                            C.byref(obj)))
    return PostsolveResult(x, y, float(obj.value))
