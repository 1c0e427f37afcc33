"""Python binding of the CPU checkers -- TEST INFRASTRUCTURE ONLY.

* ``OraclePort``: the C restatement of the reference's PDLP path
  (oracle/pdlp_oracle.c, built to oracle/build/liboracle_pdlp.so).
* ``ReferencePdlp``: the reference's own solve_pdlp / equilibrate_model /
  verify_primal / parse_mps, compiled from its sources into
  oracle/_ref/libref_pdlp.so by oracle/Makefile (absent where the reference
  sources were never available; the built library travels with the repo).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this
module, as the checker; the engine never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "markov-zip1_b200"))

from mcpdlp import _abi  # noqa: E402
from mcpdlp.model import Model  # noqa: E402
from mcpdlp.presolve import (CanonicalModel, PostsolveResult, PresolveOptions, PresolveResult,  # noqa: E402
                             PresolveStack, PresolveStatistics, SolveStatus)

ORACLE_LIB = HERE / "build" / "liboracle_pdlp.so"
REF_LIB = HERE / "_ref" / "libref_pdlp.so"
# The reference checkout: MC_REFERENCE_DIR, else the default that
# oracle/Makefile uses for REF.
REFERENCE_SOURCES = Path(os.environ.get("MC_REFERENCE_DIR", "/root/reference"))

_VP = C.c_void_p


def build(reference: bool | None = None) -> None:
    """Build the oracle port, and the reference library when its sources exist."""
    targets = ["oracle"]
    if reference is None:
        reference = (REFERENCE_SOURCES / "src" / "lp" / "first_order" / "pdlp.cpp").exists()
    if reference:
        targets.append("ref")
    subprocess.run(["make", "-C", str(HERE), f"REF={REFERENCE_SOURCES}", *targets], check=True,
                   capture_output=True)


@dataclass
class CpuSolve:
    status: int
    objective: float
    primal_infeasibility: float
    dual_infeasibility: float
    duality_gap: float
    iterations: int
    message: str
    total_ms: float
    restarts: int
    ruiz_iterations_executed: int
    primal: np.ndarray
    dual: np.ndarray
    trace: dict | None = None
    final_primal_weight: float = float("nan")


def _ptr(a):
    return None if a is None else a.ctypes.data


def _result(res: _abi.McPdlpResult, x, y, trace=None) -> CpuSolve:
    return CpuSolve(res.status, res.objective, res.primal_infeasibility,
                    res.dual_infeasibility, res.duality_gap, res.iterations,
                    res.message.decode(), res.total_ms, res.restarts,
                    res.ruiz_iterations_executed, x, y, trace, res.final_primal_weight)


def make_trace(capacity: int):
    arrays = dict(iteration=np.zeros(capacity, np.int64),
                  primal_infeasibility=np.zeros(capacity),
                  dual_infeasibility=np.zeros(capacity),
                  duality_gap=np.zeros(capacity),
                  step_size=np.zeros(capacity),
                  primal_weight=np.zeros(capacity),
                  restarted=np.zeros(capacity, np.int32))
    t = _abi.McPdlpTrace()
    t.capacity = capacity
    t.count = 0
    for k, a in arrays.items():
        setattr(t, k, a.ctypes.data)
    return t, arrays


def trace_dict(t, arrays) -> dict:
    return {k: a[: t.count].copy() for k, a in arrays.items()}


class _PresolveArrays:
    """Worst-case output arrays of a presolve of `model` (see presolve_oracle.h)."""

    def __init__(self, model: CanonicalModel):
        m, n, z = model.num_rows, model.num_cols, model.nnz
        r = m + n
        self.cs = np.zeros(n + 1, np.int32)
        self.ri = np.zeros(max(z, 1), np.int32)
        self.v = np.zeros(max(z, 1))
        self.rhs = np.zeros(max(m, 1))
        self.obj = np.zeros(max(n, 1))
        self.rmap = np.zeros(max(m, 1), np.int64)
        self.cmap = np.zeros(max(n, 1), np.int64)
        self.kind = np.zeros(max(r, 1), np.int32)
        self.index = np.zeros(max(r, 1), np.int64)
        self.var = np.zeros(max(r, 1), np.int64)
        self.val = np.zeros(max(r, 1))
        self.val2 = np.zeros(max(r, 1))
        self.ist = np.zeros(r + 1, np.int64)
        self.irow = np.zeros(max(z, 1), np.int64)
        self.icoef = np.zeros(max(z, 1))

    def pointers(self) -> list:
        return [_ptr(a) for a in (self.cs, self.ri, self.v, self.rhs, self.obj, self.rmap, self.cmap, self.kind,
                                  self.index, self.var, self.val, self.val2, self.ist, self.irow, self.icoef)]

    def result(self, info: _abi.McPresolveInfo) -> PresolveResult:
        nm, nn, nz = int(info.presolved_rows), int(info.presolved_cols), int(info.presolved_nnz)
        nr, ni = int(info.records), int(info.incident_entries)
        st = PresolveStatistics(*(int(getattr(info, f)) for f in (
            "passes_executed", "empty_rows_removed", "empty_cols_removed", "fixed_vars_removed",
            "row_singletons_removed", "original_rows", "original_cols", "presolved_rows", "presolved_cols")))
        cs = self.cs[:nn + 1].copy()
        if nn == 0:
            cs = np.zeros(1, np.int32)
        model = CanonicalModel(nm, nn, cs, self.ri[:nz].copy(), self.v[:nz].copy(), self.rhs[:nm].copy(),
                               self.obj[:nn].copy(), float(info.objective_offset))
        stack = PresolveStack(self.kind[:nr].copy(), self.index[:nr].copy(), self.var[:nr].copy(),
                              self.val[:nr].copy(), self.val2[:nr].copy(), self.ist[:nr + 1].copy(),
                              self.irow[:ni].copy(), self.icoef[:ni].copy(), self.rmap[:nm].copy(),
                              self.cmap[:nn].copy())
        return PresolveResult(SolveStatus(info.status), model, stack, st, info.message.decode(),
                              dict(presolved_nnz=nz, incident_entries=ni))


class OraclePort:
    def __init__(self) -> None:
        if not ORACLE_LIB.exists():
            build(reference=False)
        lib = C.CDLL(str(ORACLE_LIB))
        lib.oracle_solve_pdlp.argtypes = [_VP] * 8
        lib.oracle_solve_pdlp.restype = C.c_int
        lib.oracle_equilibrate.argtypes = [C.c_int32, C.c_int32] + [_VP] * 8 + [
            C.c_int64, C.c_double, _VP, _VP, _VP, _VP]
        lib.oracle_equilibrate.restype = C.c_int
        lib.oracle_spmv.argtypes = [C.c_int32, C.c_int32] + [_VP] * 5
        lib.oracle_spmv.restype = None
        lib.oracle_spmv_t.argtypes = [C.c_int32, C.c_int32] + [_VP] * 5
        lib.oracle_spmv_t.restype = None
        lib.oracle_presolve.argtypes = [_VP, _VP, _VP, _VP]
        lib.oracle_presolve.restype = C.c_int
        lib.oracle_postsolve.argtypes = [_VP, C.c_int64] + [_VP] * 5 + [C.c_int64, _VP, C.c_int64, _VP, _VP,
                                                                       C.c_int64, _VP, C.c_int64, _VP, _VP, _VP]
        lib.oracle_postsolve.restype = C.c_int
        self.lib = lib

    def solve(self, model: Model, options: _abi.McPdlpOptions, warm_x=None, warm_y=None,
              trace_capacity: int = 0) -> CpuSolve:
        lp = model.to_struct()
        x = np.zeros(model.num_cols)
        y = np.zeros(model.num_rows)
        res = _abi.McPdlpResult()
        tr, arrays = make_trace(trace_capacity) if trace_capacity else (None, None)
        rc = self.lib.oracle_solve_pdlp(C.addressof(lp), C.addressof(options), _ptr(warm_x),
                                        _ptr(warm_y), _ptr(x), _ptr(y), C.addressof(res),
                                        C.addressof(tr) if tr is not None else None)
        if rc != 0:
            raise RuntimeError(f"oracle_solve_pdlp failed ({rc})")
        return _result(res, x, y, trace_dict(tr, arrays) if tr is not None else None)

    def equilibrate(self, model: Model, max_iterations: int = 10):
        v = model.value.copy()
        obj = model.objective.copy()
        vl, vu = model.var_lower.copy(), model.var_upper.copy()
        rl, ru = model.row_lower.copy(), model.row_upper.copy()
        rs = np.zeros(model.num_rows)
        cs = np.zeros(model.num_cols)
        it = C.c_int64(0)
        conv = C.c_int32(0)
        rc = self.lib.oracle_equilibrate(model.num_rows, model.num_cols, _ptr(model.col_start),
                                         _ptr(model.row_index), _ptr(v), _ptr(obj), _ptr(vl),
                                         _ptr(vu), _ptr(rl), _ptr(ru), max_iterations, 1e-3,
                                         _ptr(rs), _ptr(cs), C.addressof(it), C.addressof(conv))
        if rc != 0:
            raise RuntimeError("oracle_equilibrate failed")
        return dict(value=v, objective=obj, var_lower=vl, var_upper=vu, row_lower=rl,
                    row_upper=ru, row_scale=rs, col_scale=cs, iterations=it.value,
                    converged=bool(conv.value))

    def spmv(self, model: Model, x: np.ndarray) -> np.ndarray:
        y = np.zeros(model.num_rows)
        self.lib.oracle_spmv(model.num_rows, model.num_cols, _ptr(model.col_start),
                             _ptr(model.row_index), _ptr(model.value), _ptr(x), _ptr(y))
        return y

    def spmv_t(self, model: Model, y: np.ndarray) -> np.ndarray:
        z = np.zeros(model.num_cols)
        self.lib.oracle_spmv_t(model.num_rows, model.num_cols, _ptr(model.col_start),
                               _ptr(model.row_index), _ptr(model.value), _ptr(y), _ptr(z))
        return z

    def presolve(self, model: CanonicalModel, options: PresolveOptions | None = None) -> PresolveResult:
        """The restated presolve (presolve_oracle.c); ValueError where the
        reference's validate() throws."""
        o = (options or PresolveOptions()).to_struct()
        s = model.to_struct()
        arr = _PresolveArrays(model)
        out = (C.c_void_p * 15)(*arr.pointers())
        info = _abi.McPresolveInfo()
        rc = self.lib.oracle_presolve(C.addressof(s), C.addressof(o), C.addressof(info), C.addressof(out))
        if rc == _abi.MC_ERR_INVALID_ARGUMENT:
            raise ValueError("oracle_presolve: invalid canonical model")
        if rc != 0:
            raise RuntimeError(f"oracle_presolve failed ({rc})")
        return arr.result(info)

    def postsolve(self, res: PresolveResult, model: CanonicalModel, primal: np.ndarray,
                  dual: np.ndarray) -> PostsolveResult:
        st = res.stack
        rx = np.ascontiguousarray(primal, dtype=np.float64)
        ry = np.ascontiguousarray(dual, dtype=np.float64)
        x, y, obj = np.zeros(model.num_cols), np.zeros(model.num_rows), C.c_double()
        s = model.to_struct()
        rc = self.lib.oracle_postsolve(C.addressof(s), st.size(), _ptr(st.kind), _ptr(st.index), _ptr(st.variable),
                                       _ptr(st.value), _ptr(st.value2), len(st.presolved_to_original_rows),
                                       _ptr(st.presolved_to_original_rows), len(st.presolved_to_original_cols),
                                       _ptr(st.presolved_to_original_cols), _ptr(rx), len(rx), _ptr(ry), len(ry),
                                       _ptr(x), _ptr(y), C.addressof(obj))
        if rc != 0:
            raise ValueError(f"oracle_postsolve failed ({rc})")
        return PostsolveResult(x, y, obj.value)


class ReferencePdlp:
    """The reference's compiled CPU code; ``available()`` is False if not built."""

    @staticmethod
    def available() -> bool:
        return REF_LIB.exists()

    def __init__(self) -> None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} is not built")
        lib = C.CDLL(str(REF_LIB))
        lib.ref_solve_pdlp.argtypes = [_VP] * 5
        lib.ref_solve_pdlp.restype = C.c_int
        lib.ref_equilibrate_model.argtypes = [_VP, C.c_int64] + [_VP] * 10
        lib.ref_equilibrate_model.restype = C.c_int
        lib.ref_verify_primal.argtypes = [_VP, _VP, C.c_double, C.c_double, _VP, _VP, _VP, _VP]
        lib.ref_verify_primal.restype = C.c_int
        lib.ref_mps_load.argtypes = [C.c_char_p, _VP, _VP, _VP, _VP, _VP]
        lib.ref_mps_load.restype = C.c_int
        lib.ref_mps_fetch.argtypes = [_VP] * 8
        lib.ref_mps_fetch.restype = C.c_int
        lib.ref_last_error.argtypes = [C.c_char_p, C.c_size_t]
        lib.ref_last_error.restype = C.c_int
        lib.ref_verify_primal_report.argtypes = [_VP, _VP] + [C.c_double] * 5 + [_VP] * 4
        lib.ref_verify_primal_report.restype = C.c_int
        lib.ref_canonical_sizes.argtypes = [_VP, _VP, _VP, _VP]
        lib.ref_canonical_sizes.restype = C.c_int
        lib.ref_canonical_equilibrate.argtypes = [C.c_int64] + [C.c_double] * 3 + [_VP] * 14
        lib.ref_canonical_equilibrate.restype = C.c_int
        lib.ref_simplex_solve.argtypes = [_VP, C.c_int64, _VP, _VP, _VP, _VP]
        lib.ref_simplex_solve.restype = C.c_int
        lib.ref_canonical_fetch.argtypes = [_VP] * 6
        lib.ref_canonical_fetch.restype = C.c_int
        lib.ref_presolve.argtypes = [_VP, _VP, _VP]
        lib.ref_presolve.restype = C.c_int
        lib.ref_presolve_fetch.argtypes = [_VP] * 15
        lib.ref_presolve_fetch.restype = C.c_int
        lib.ref_postsolve.argtypes = [_VP, C.c_int64, _VP, C.c_int64, _VP, _VP, _VP]
        lib.ref_postsolve.restype = C.c_int
        self.lib = lib

    def _err(self) -> str:
        b = C.create_string_buffer(512)
        self.lib.ref_last_error(b, 512)
        return b.value.decode()

    def solve(self, model: Model, options: _abi.McPdlpOptions) -> CpuSolve:
        lp = model.to_struct()
        x = np.zeros(model.num_cols)
        y = np.zeros(model.num_rows)
        res = _abi.McPdlpResult()
        rc = self.lib.ref_solve_pdlp(C.addressof(lp), C.addressof(options), _ptr(x), _ptr(y),
                                     C.addressof(res))
        if rc != 0:
            raise RuntimeError(f"reference solve_pdlp threw: {self._err()}")
        return _result(res, x, y)

    def equilibrate(self, model: Model, max_iterations: int = 10):
        lp = model.to_struct()
        v = np.zeros(model.nnz)
        obj = np.zeros(model.num_cols)
        vl, vu = np.zeros(model.num_cols), np.zeros(model.num_cols)
        rl, ru = np.zeros(model.num_rows), np.zeros(model.num_rows)
        rs, cs = np.zeros(model.num_rows), np.zeros(model.num_cols)
        it = C.c_int64(0)
        conv = C.c_int32(0)
        rc = self.lib.ref_equilibrate_model(C.addressof(lp), max_iterations, _ptr(v), _ptr(obj),
                                            _ptr(vl), _ptr(vu), _ptr(rl), _ptr(ru), _ptr(rs),
                                            _ptr(cs), C.addressof(it), C.addressof(conv))
        if rc != 0:
            raise RuntimeError(f"reference equilibrate_model threw: {self._err()}")
        return dict(value=v, objective=obj, var_lower=vl, var_upper=vu, row_lower=rl,
                    row_upper=ru, row_scale=rs, col_scale=cs, iterations=it.value,
                    converged=bool(conv.value))

    SIMPLEX_STATUS = ("optimal", "infeasible", "unbounded", "iteration_limit", "invalid_model",
                      "invalid_options", "resource_limit", "numerical_failure")

    def simplex(self, model: Model, iteration_limit: int = 0) -> dict:
        """The reference's primal simplex (src/lp/reference/revised_simplex.cpp)
        on a small LP, through the CLI's canonical path: the FP64 optimum of
        LPs the simplex's dense limits admit (canonical rows <= 1024)."""
        lp = model.to_struct()
        x = np.zeros(model.num_cols)
        obj = C.c_double(np.nan)
        st = C.c_int32(-1)
        it = C.c_int64(0)
        rc = self.lib.ref_simplex_solve(C.addressof(lp), iteration_limit, _ptr(x), C.addressof(obj),
                                        C.addressof(st), C.addressof(it))
        if rc != 0:
            raise RuntimeError(f"reference simplex threw: {self._err()}")
        return dict(status=self.SIMPLEX_STATUS[st.value], objective=obj.value, primal=x,
                    iterations=it.value)

    KINDS = ("variable_lower", "variable_upper", "row_lower", "row_upper", "objective")

    def verify_report(self, model: Model, primal: np.ndarray, claimed: float, feasibility_tolerance: float,
                      objective_tolerance: float) -> dict:
        """The reference verify_primal's full report (counts and lowest index
        per violation category), absolute = relative tolerance per kind."""
        lp = model.to_struct()
        x = np.ascontiguousarray(primal, dtype=np.float64)
        counts = np.zeros(5, np.int64)
        first = np.zeros(5, np.int64)
        out = np.zeros(4)
        passed = C.c_int32(0)
        ft, ot = feasibility_tolerance, objective_tolerance
        rc = self.lib.ref_verify_primal_report(C.addressof(lp), _ptr(x), claimed, ft, ft, ot, ot, _ptr(counts),
                                               _ptr(first), _ptr(out), C.addressof(passed))
        if rc != 0:
            raise RuntimeError(f"reference verify_primal threw: {self._err()}")
        return dict(passed=bool(passed.value), recomputed_objective=out[0], objective_difference=out[1],
                    maximum_row_violation=out[2], maximum_variable_violation=out[3],
                    violations={k: int(counts[q]) for q, k in enumerate(self.KINDS)},
                    first_index={k: int(first[q]) for q, k in enumerate(self.KINDS)})

    def canonical_equilibrate(self, model: Model, max_iterations: int = 10, tolerance: float = 1e-3,
                              min_scale: float = 1e-4, max_scale: float = 1e4) -> dict:
        """The CLI's canonical model of `model` (sparse_canonicalize) before and
        after the reference's equilibrate (src/scale/ruiz_scaling.cpp:20-125)."""
        lp = model.to_struct()
        m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
        if self.lib.ref_canonical_sizes(C.addressof(lp), C.addressof(m), C.addressof(n), C.addressof(z)) != 0:
            raise RuntimeError(f"reference sparse_canonicalize threw: {self._err()}")
        m, n, z = m.value, n.value, z.value
        out = dict(m=m, n=n, nnz=z, col_start=np.zeros(n + 1, np.int32), row_index=np.zeros(z, np.int32))
        for k, size in (("value_in", z), ("rhs_in", m), ("objective_in", n), ("value", z), ("rhs", m),
                        ("objective", n), ("row_scale", m), ("col_scale", n), ("inv_row_scale", m),
                        ("inv_col_scale", n)):
            out[k] = np.zeros(size)
        it, conv = C.c_int64(), C.c_int32()
        rc = self.lib.ref_canonical_equilibrate(
            max_iterations, tolerance, min_scale, max_scale, _ptr(out["col_start"]), _ptr(out["row_index"]),
            _ptr(out["value_in"]), _ptr(out["rhs_in"]), _ptr(out["objective_in"]), _ptr(out["value"]),
            _ptr(out["rhs"]), _ptr(out["objective"]), _ptr(out["row_scale"]), _ptr(out["col_scale"]),
            _ptr(out["inv_row_scale"]), _ptr(out["inv_col_scale"]), C.addressof(it), C.addressof(conv))
        if rc != 0:
            raise RuntimeError(f"reference equilibrate threw: {self._err()}")
        out["iterations"], out["converged"] = it.value, bool(conv.value)
        return out

    def verify_primal(self, model: Model, primal: np.ndarray, claimed: float, tol: float):
        lp = model.to_struct()
        passed = C.c_int32(0)
        rv, vv, ro = C.c_double(0), C.c_double(0), C.c_double(0)
        rc = self.lib.ref_verify_primal(C.addressof(lp), _ptr(np.ascontiguousarray(primal)),
                                        claimed, tol, C.addressof(passed), C.addressof(rv),
                                        C.addressof(vv), C.addressof(ro))
        if rc != 0:
            raise RuntimeError(f"reference verify_primal threw: {self._err()}")
        return dict(passed=bool(passed.value), max_row_violation=rv.value,
                    max_var_violation=vv.value, recomputed_objective=ro.value)

    def parse_mps(self, path: str | Path) -> Model:
        m, n, s = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        nnz = C.c_int64(0)
        off = C.c_double(0)
        rc = self.lib.ref_mps_load(str(path).encode(), C.addressof(m), C.addressof(n),
                                   C.addressof(nnz), C.addressof(s), C.addressof(off))
        if rc != 0:
            raise RuntimeError(f"reference parse_mps threw: {self._err()}")
        M, N, Z = m.value, n.value, nnz.value
        cs = np.zeros(N + 1, np.int32)
        ri = np.zeros(Z, np.int32)
        v = np.zeros(Z)
        obj, vl, vu = np.zeros(N), np.zeros(N), np.zeros(N)
        rl, ru = np.zeros(M), np.zeros(M)
        self.lib.ref_mps_fetch(_ptr(cs), _ptr(ri), _ptr(v), _ptr(obj), _ptr(vl), _ptr(vu),
                               _ptr(rl), _ptr(ru))
        return Model(M, N, cs, ri, v, obj, vl, vu, rl, ru, off.value, s.value,
                     name=Path(path).stem)

    def canonical_model(self, model: Model) -> CanonicalModel:
        """The CLI's canonical model of `model` (sparse_canonicalize,
        src/transform/sparse_canonicalize.cpp), unscaled."""
        lp = model.to_struct()
        m, n, z = C.c_int64(), C.c_int64(), C.c_int64()
        if self.lib.ref_canonical_sizes(C.addressof(lp), C.addressof(m), C.addressof(n), C.addressof(z)) != 0:
            raise RuntimeError(f"reference sparse_canonicalize threw: {self._err()}")
        m, n, z = m.value, n.value, z.value
        cs, ri, v = np.zeros(n + 1, np.int32), np.zeros(max(z, 1), np.int32), np.zeros(max(z, 1))
        rhs, obj, off = np.zeros(max(m, 1)), np.zeros(max(n, 1)), C.c_double()
        self.lib.ref_canonical_fetch(_ptr(cs), _ptr(ri), _ptr(v), _ptr(rhs), _ptr(obj), C.addressof(off))
        return CanonicalModel(m, n, cs, ri[:z], v[:z], rhs[:m], obj[:n], off.value)

    def presolve(self, model: CanonicalModel, options: PresolveOptions | None = None) -> PresolveResult:
        """The reference's presolve (src/presolve/presolve.cpp:20); keeps its
        result for postsolve().  ValueError where it throws."""
        o = (options or PresolveOptions()).to_struct()
        s = model.to_struct()
        info = _abi.McPresolveInfo()
        if self.lib.ref_presolve(C.addressof(s), C.addressof(o), C.addressof(info)) != 0:
            raise ValueError(f"reference presolve threw: {self._err()}")
        arr = _PresolveArrays(model)
        self.lib.ref_presolve_fetch(*arr.pointers())
        return arr.result(info)

    def postsolve(self, model: CanonicalModel, primal: np.ndarray, dual: np.ndarray) -> PostsolveResult:
        """postsolve() of the last presolve() against its input model."""
        rx = np.ascontiguousarray(primal, dtype=np.float64)
        ry = np.ascontiguousarray(dual, dtype=np.float64)
        x, y, obj = np.zeros(max(model.num_cols, 1)), np.zeros(max(model.num_rows, 1)), C.c_double()
        if self.lib.ref_postsolve(_ptr(rx), len(rx), _ptr(ry), len(ry), _ptr(x), _ptr(y), C.addressof(obj)) != 0:
            raise ValueError(f"reference postsolve threw: {self._err()}")
        return PostsolveResult(x[:model.num_cols], y[:model.num_rows], obj.value)


def presolve_mismatch(a: PresolveResult, b: PresolveResult) -> str | None:
    """The first field in which two presolve results differ (bit for bit),
    or None if they are identical."""
    if a.status != b.status or a.message != b.message:
        return f"status/message {a.status}:{a.message!r} vs {b.status}:{b.message!r}"
    if a.statistics != b.statistics:
        return f"statistics {a.statistics} vs {b.statistics}"
    if (a.model.num_rows, a.model.num_cols) != (b.model.num_rows, b.model.num_cols):
        return "reduced model shape"
    if a.model.objective_offset != b.model.objective_offset:
        return f"objective offset {a.model.objective_offset!r} vs {b.model.objective_offset!r}"
    for f in ("col_start", "row_index", "value", "rhs", "objective"):
        if not np.array_equal(getattr(a.model, f), getattr(b.model, f)):
            return f"reduced model {f}"
    for f in ("kind", "index", "variable", "value", "value2", "incident_start", "incident_row",
              "incident_coefficient", "presolved_to_original_rows", "presolved_to_original_cols"):
        if not np.array_equal(getattr(a.stack, f), getattr(b.stack, f)):
            return f"stack {f}"
    return None
