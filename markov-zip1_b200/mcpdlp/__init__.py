"""B200 PDLP engine: Python mirror of the reference's first-order LP interface.

Same names, fields, defaults and statuses as the reference C++ API
(include/markov_cero/lp/first_order/pdlp.hpp):

    PdlpOptions   pdlp.hpp:18-41      PdlpStatus    pdlp.hpp:43
    PdlpResult    pdlp.hpp:45-63      solve_pdlp    pdlp.hpp:67 / pdlp.cpp:139

``solve_pdlp`` runs the CUDA engine (lib/libmcpdlp.so) through its C ABI
(include/mc_pdlp.h).  There is no CPU path: ``Backend.cpu`` is rejected, a
missing library raises ``EngineUnavailable`` and a machine without an sm_100
device raises ``EngineError`` (no_device).  Errors keep the reference's
classes: malformed models raise ``ValueError`` (std::invalid_argument),
size limits raise ``EngineError`` with code resource_limit.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field, fields
from typing import Optional

import numpy as np

from . import _abi, _lib
from ._lib import EngineError, EngineUnavailable, build, engine, engine_built
from .model import Model, ObjectiveSense, from_triplets

__all__ = [
    "Backend", "RestartStrategy", "PdlpStatus", "Precision", "PdlpOptions", "PdlpResult",
    "Model", "ObjectiveSense", "Context", "solve_pdlp", "EngineError", "EngineUnavailable",
    "from_triplets", "device_count", "build", "engine_built", "StepwiseSolve", "DeviceModel",
]


class Backend(enum.IntEnum):          # pdlp.hpp:15
    cpu = 0
    gpu = 1


class RestartStrategy(enum.IntEnum):  # pdlp.hpp:16
    none = 0
    adaptive = 1
    fixed = 2


class PdlpStatus(enum.IntEnum):       # pdlp.hpp:43
    optimal = 0
    iteration_limit = 1
    infeasible_or_unbounded = 2
    numerical_failure = 3


class Precision(enum.IntEnum):        # engine extension
    fp64 = 0
    fp32_refine = 1


@dataclass
class PdlpOptions:
    """PdlpOptions (pdlp.hpp:18-41) plus the engine's extensions."""
    max_iterations: int = 100000
    restart_every: int = 40
    primal_tolerance: float = 1e-4
    dual_tolerance: float = 1e-4
    gap_tolerance: float = 1e-4
    step_size_reduction: float = 0.9
    power_iterations: int = 20
    backend: Backend = Backend.gpu
    restart_strategy: RestartStrategy = RestartStrategy.adaptive
    restart_reduction_factor: float = 0.368
    adaptive_step_size: bool = True
    adaptive_primal_weight: bool = True
    initial_primal_weight: float = 0.0
    primal_weight_smoothing: float = 0.5
    ruiz_scaling: bool = True
    ruiz_iterations: int = 10
    # ---- extensions (no counterpart in the reference) ----
    precision: Precision = Precision.fp64
    device: int = 0
    profile_kernels: bool = False
    check_every_chunks: int = 1
    lanes_per_column: int = 0                      # SpMV tuning, 0 = chosen by line length
    lanes_per_row: int = 0
    warm_start_guard: bool = False                 # run from the better of warm / cold start
    initial_primal: Optional[np.ndarray] = None   # warm start, original space
    initial_dual: Optional[np.ndarray] = None

    def set_tolerance(self, tol: float) -> None:
        """pdlp.hpp:35-39"""
        self.primal_tolerance = tol
        self.dual_tolerance = tol
        self.gap_tolerance = tol

    def to_struct(self) -> _abi.McPdlpOptions:
        if self.backend != Backend.gpu:
            raise ValueError("this engine runs PDLP on the GPU only (Backend.gpu); "
                             "Backend.cpu is the reference solver's own path")
        o = _abi.default_options_struct()
        for f in fields(self):
            if f.name in ("initial_primal", "initial_dual"):
                continue
            v = getattr(self, f.name)
            setattr(o, f.name, int(v) if isinstance(v, (bool, enum.IntEnum)) else v)
        return o


@dataclass
class PdlpResult:
    """PdlpResult (pdlp.hpp:45-63) plus ``extra`` engine counters."""
    status: PdlpStatus = PdlpStatus.iteration_limit
    primal: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dual: np.ndarray = field(default_factory=lambda: np.zeros(0))
    objective: float = 0.0
    primal_infeasibility: float = 0.0
    dual_infeasibility: float = 0.0
    duality_gap: float = 0.0
    tolerance: float = 1e-4
    iterations: int = 0
    message: str = ""
    h2d_ms: float = 0.0
    kernel_ms: float = 0.0
    d2h_ms: float = 0.0
    total_ms: float = 0.0
    backend_actually_used: str = "cuda"
    extra: dict = field(default_factory=dict)
    trace: Optional[dict] = None


def _result_from(r: _abi.McPdlpResult, x, y, trace=None) -> PdlpResult:
    extra = dict(
        ruiz_iterations_executed=r.ruiz_iterations_executed,
        restarts=r.restarts,
        final_primal_weight=r.final_primal_weight,
        final_step_size=r.final_step_size,
        refinement_rounds=r.refinement_rounds,
        inner_iterations=r.inner_iterations,
        kernel_launches=r.kernel_launches,
        warm_start_used=bool(r.warm_start_used),
        warm_start_score=r.warm_start_score,
        cold_start_score=r.cold_start_score,
        certificate=_abi.CERTIFICATE_NAMES[r.certificate] if 0 <= r.certificate < 4 else str(r.certificate),
        certificate_index=r.certificate_index,
        launches_by_kind={n: r.launches_by_kind[i] for i, n in enumerate(_abi.KERNEL_KIND_NAMES)
                          if n != "-"},
        kernel_ms_by_kind={n: r.kernel_ms_by_kind[i] for i, n in enumerate(_abi.KERNEL_KIND_NAMES)
                           if n != "-"},
    )
    return PdlpResult(PdlpStatus(r.status), x, y, r.objective, r.primal_infeasibility,
                      r.dual_infeasibility, r.duality_gap, r.tolerance, r.iterations,
                      r.message.decode(errors="replace"), r.h2d_ms, r.kernel_ms, r.d2h_ms,
                      r.total_ms, r.backend_actually_used.decode(), extra, trace)


def _make_trace(capacity: int):
    arrays = dict(iteration=np.zeros(capacity, np.int64), primal_infeasibility=np.zeros(capacity),
                  dual_infeasibility=np.zeros(capacity), duality_gap=np.zeros(capacity),
                  step_size=np.zeros(capacity), primal_weight=np.zeros(capacity),
                  restarted=np.zeros(capacity, np.int32))
    t = _abi.McPdlpTrace()
    t.capacity = capacity
    for k, a in arrays.items():
        setattr(t, k, a.ctypes.data)
    return t, arrays


def device_count() -> int:
    n = C.c_int(0)
    _lib.check(engine().mc_device_count(C.byref(n)))
    return n.value


def _raise(code: int) -> None:
    if code == _abi.MC_ERR_INVALID_ARGUMENT:
        raise ValueError(_lib.last_error())
    _lib.check(code)


class Context:
    """A device, a stream and reusable device buffers (mc_pdlp_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = engine()
        self._h = C.c_void_p()
        _raise(self._lib.mc_pdlp_ctx_create(device, C.byref(self._h)))
        self.device = device

    def close(self) -> None:
        if self._h:
            self._lib.mc_pdlp_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (every engine kernel of
        this context runs on it; torch.cuda.ExternalStream wraps it)."""
        p = C.c_void_p()
        _raise(self._lib.mc_pdlp_ctx_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def solve(self, model: Model, options: Optional[PdlpOptions] = None,
              trace_capacity: int = 0) -> PdlpResult:
        """solve_pdlp on host arrays (copies in and out are part of the call)."""
        options = options or PdlpOptions()
        o = options.to_struct()
        lp = model.to_struct()
        x = np.zeros(model.num_cols)
        y = np.zeros(model.num_rows)
        wx = None if options.initial_primal is None else np.ascontiguousarray(options.initial_primal, np.float64)
        wy = None if options.initial_dual is None else np.ascontiguousarray(options.initial_dual, np.float64)
        if wx is not None and len(wx) != model.num_cols:
            raise ValueError("initial_primal has the wrong length")
        if wy is not None and len(wy) != model.num_rows:
            raise ValueError("initial_dual has the wrong length")
        res = _abi.McPdlpResult()
        tr, arrays = _make_trace(trace_capacity) if trace_capacity > 0 else (None, None)
        rc = self._lib.mc_pdlp_ctx_solve(
            self._h, C.addressof(lp), C.addressof(o),
            None if wx is None else wx.ctypes.data, None if wy is None else wy.ctypes.data,
            x.ctypes.data, y.ctypes.data, C.addressof(res),
            C.addressof(tr) if tr is not None else None)
        _raise(rc)
        trace = {k: a[: tr.count].copy() for k, a in arrays.items()} if tr is not None else None
        if model.num_rows == 0 or model.num_cols == 0:
            x, y = np.zeros(0), np.zeros(0)
        return _result_from(res, x, y, trace)

    def begin(self, model, options: Optional[PdlpOptions] = None,
              trace_capacity: int = 0) -> "StepwiseSolve":
        """Start a stepwise solve (mc_pdlp_ctx_begin) of a host Model or a
        DeviceModel: everything before the first iteration.  Drive it with
        ``iterate(chunks)`` and end it with ``finish()``; the result equals
        ``solve`` / ``solve_device`` with the same options."""
        return StepwiseSolve(self, model, options or PdlpOptions(), trace_capacity)

    def solve_batch(self, models: list, options: Optional[PdlpOptions] = None,
                    initial_primal: Optional[list] = None, initial_dual: Optional[list] = None) -> list:
        """Solve many independent LPs together (mc_pdlp_ctx_solve_batch): one
        PdlpResult per model, each from its own run of the algorithm.  With
        initial_primal / initial_dual (lists with an array or None per model)
        each LP starts from its given point (mc_pdlp_ctx_solve_batch_warm)."""
        options = options or PdlpOptions()
        o = options.to_struct()
        count = len(models)
        lps = (_abi.McLp * count)()
        xs = [np.zeros(mm.num_cols) for mm in models]
        ys = [np.zeros(mm.num_rows) for mm in models]
        for b, mm in enumerate(models):
            lps[b] = mm.to_struct()
        xp = (C.c_void_p * count)(*[a.ctypes.data if len(a) else None for a in xs])
        yp = (C.c_void_p * count)(*[a.ctypes.data if len(a) else None for a in ys])
        res = (_abi.McPdlpResult * count)()
        if initial_primal is None and initial_dual is None:
            _raise(self._lib.mc_pdlp_ctx_solve_batch(self._h, C.addressof(lps), count, C.addressof(o),
                                                     C.addressof(xp), C.addressof(yp), C.addressof(res)))
        else:
            keep = []

            def starts(given, sizes):
                out = (C.c_void_p * count)()
                for b in range(count):
                    v = None if given is None else given[b]
                    if v is not None:
                        a = np.ascontiguousarray(v, dtype=np.float64)
                        if a.shape != (sizes[b],):
                            raise ValueError("starting point dimension mismatch")
                        keep.append(a)
                        out[b] = a.ctypes.data
                return out
            x0 = starts(initial_primal, [mm.num_cols for mm in models])
            y0 = starts(initial_dual, [mm.num_rows for mm in models])
            _raise(self._lib.mc_pdlp_ctx_solve_batch_warm(self._h, C.addressof(lps), count, C.addressof(o),
                                                          C.addressof(x0), C.addressof(y0), C.addressof(xp),
                                                          C.addressof(yp), C.addressof(res)))
        return [_result_from(res[b], xs[b], ys[b]) for b in range(count)]

    def solve_variants(self, base: Model, var_lower: list, var_upper: list,
                       options: Optional[PdlpOptions] = None, initial_primal: Optional[list] = None,
                       initial_dual: Optional[list] = None) -> list:
        """Solve variants of `base` that differ only in their variable bounds
        (mc_pdlp_ctx_solve_variants): var_lower[b] / var_upper[b] are arrays
        of num_cols (None keeps the base's).  One PdlpResult per variant."""
        options = options or PdlpOptions()
        o = options.to_struct()
        count = len(var_lower)
        if len(var_upper) != count or count == 0:
            raise ValueError("var_lower and var_upper need one entry per variant")
        n, m = base.num_cols, base.num_rows
        keep = []

        def ptrs(given, size):
            out = (C.c_void_p * count)()
            for b in range(count):
                v = None if given is None else given[b]
                if v is not None:
                    a = np.ascontiguousarray(v, dtype=np.float64)
                    if a.shape != (size,):
                        raise ValueError("variant array dimension mismatch")
                    keep.append(a)
                    out[b] = a.ctypes.data
            return out
        lo, hi = ptrs(var_lower, n), ptrs(var_upper, n)
        x0, y0 = ptrs(initial_primal, n), ptrs(initial_dual, m)
        xs = [np.zeros(n) for _ in range(count)]
        ys = [np.zeros(m) for _ in range(count)]
        xp = (C.c_void_p * count)(*[a.ctypes.data if len(a) else None for a in xs])
        yp = (C.c_void_p * count)(*[a.ctypes.data if len(a) else None for a in ys])
        res = (_abi.McPdlpResult * count)()
        lp = base.to_struct()
        _raise(self._lib.mc_pdlp_ctx_solve_variants(self._h, C.addressof(lp), count, C.addressof(lo),
                                                    C.addressof(hi), C.addressof(o), C.addressof(x0),
                                                    C.addressof(y0), C.addressof(xp), C.addressof(yp),
                                                    C.addressof(res)))
        return [_result_from(res[b], xs[b], ys[b]) for b in range(count)]

    def verify_primal(self, model: Model, primal, claimed_objective: float,
                      feasibility_tolerance: float = 1e-7, objective_tolerance: float = 1e-7) -> dict:
        """verify_primal (src/verify/primal_verifier.cpp:44) on the device
        (mc_verify_primal): absolute and relative tolerance both set to the
        given value per kind, as the CLI does after a PDLP solve."""
        lp = model.to_struct()
        x = np.ascontiguousarray(primal, dtype=np.float64)
        if x.shape != (model.num_cols,):
            raise ValueError("candidate dimension mismatch")
        rep = _abi.McVerifyReport()
        _raise(self._lib.mc_verify_primal(self._h, C.addressof(lp), x.ctypes.data, float(claimed_objective),
                                          feasibility_tolerance, feasibility_tolerance, objective_tolerance,
                                          objective_tolerance, C.addressof(rep)))
        return dict(passed=bool(rep.passed), recomputed_objective=rep.recomputed_objective,
                    objective_difference=rep.objective_difference,
                    maximum_row_violation=rep.maximum_row_violation,
                    maximum_variable_violation=rep.maximum_variable_violation,
                    violations={k: int(rep.violations[q]) for q, k in enumerate(_abi.VIOLATION_KINDS)},
                    first_index={k: int(rep.first_index[q]) for q, k in enumerate(_abi.VIOLATION_KINDS)})

    def solve_device(self, dlp: "DeviceModel", options: Optional[PdlpOptions] = None,
                     primal_out=None, dual_out=None) -> PdlpResult:
        """solve_pdlp on a device-resident model (torch CUDA tensors); the
        unscaled averages are written to primal_out / dual_out (device).
        options.initial_primal / initial_dual, when given, must be torch CUDA
        tensors on the model's device (float64, n and m entries)."""
        options = options or PdlpOptions()
        o = options.to_struct()
        lp = dlp.to_struct()
        res = _abi.McPdlpResult()
        starts = []
        for v, size in ((options.initial_primal, dlp.num_cols), (options.initial_dual, dlp.num_rows)):
            if v is None:
                starts.append(None)
                continue
            if not hasattr(v, "data_ptr") or not getattr(v, "is_cuda", False):
                raise ValueError("a device model takes device (torch CUDA) starting points")
            if tuple(v.shape) != (size,) or str(v.dtype) != "torch.float64" or not v.is_contiguous():
                raise ValueError("starting point must be a contiguous float64 tensor of the model's size")
            starts.append(v.data_ptr())
        rc = self._lib.mc_pdlp_ctx_solve(
            self._h, C.addressof(lp), C.addressof(o), starts[0], starts[1],
            None if primal_out is None else primal_out.data_ptr(),
            None if dual_out is None else dual_out.data_ptr(), C.addressof(res), None)
        _raise(rc)
        return _result_from(res, primal_out, dual_out)


class StepwiseSolve:
    """A solve driven a few restart chunks at a time (mc_pdlp_ctx_begin /
    _iterate / _finish).  Host models are copied in at begin; a DeviceModel
    must stay alive until finish, and its outputs are device tensors."""

    def __init__(self, ctx: Context, model, options: PdlpOptions, trace_capacity: int = 0):
        self.ctx = ctx
        self.model = model
        self.device = isinstance(model, DeviceModel)
        self._lp = model.to_struct()
        self._opts = options.to_struct()
        self._keep = []
        warm = []
        for a, size in ((options.initial_primal, model.num_cols), (options.initial_dual, model.num_rows)):
            if a is None:
                warm.append(None)
            elif self.device:
                warm.append(a.data_ptr())
                self._keep.append(a)
            else:
                arr = np.ascontiguousarray(a, np.float64)
                if arr.shape != (size,):
                    raise ValueError("starting point dimension mismatch")
                self._keep.append(arr)
                warm.append(arr.ctypes.data)
        self._trace, self._trace_arrays = (_make_trace(trace_capacity) if trace_capacity > 0
                                           else (None, None))
        _raise(ctx._lib.mc_pdlp_ctx_begin(ctx.handle, C.addressof(self._lp), C.addressof(self._opts),
                                          warm[0], warm[1],
                                          C.addressof(self._trace) if self._trace is not None else None))
        self.iterations = 0
        self.finished = False

    def iterate(self, chunks: int = 1) -> tuple[int, bool]:
        """Up to `chunks` further restart chunks; (iterations so far, finished)."""
        it = C.c_int64(0)
        fin = C.c_int32(0)
        _raise(self.ctx._lib.mc_pdlp_ctx_iterate(self.ctx.handle, int(chunks), C.byref(it), C.byref(fin)))
        self.iterations, self.finished = int(it.value), bool(fin.value)
        return self.iterations, self.finished

    def finish(self, primal_out=None, dual_out=None) -> PdlpResult:
        """Outputs and result (mc_pdlp_ctx_finish).  Host models: numpy arrays
        are returned; device models: pass device tensors (or None)."""
        res = _abi.McPdlpResult()
        m = self.model
        if self.device:
            x, y = primal_out, dual_out
            xp = None if x is None else x.data_ptr()
            yp = None if y is None else y.data_ptr()
        else:
            x, y = np.zeros(m.num_cols), np.zeros(m.num_rows)
            xp, yp = x.ctypes.data, y.ctypes.data
        _raise(self.ctx._lib.mc_pdlp_ctx_finish(self.ctx.handle, xp, yp, C.addressof(res)))
        tr = self._trace
        trace = ({k: a[: tr.count].copy() for k, a in self._trace_arrays.items()}
                 if tr is not None else None)
        if not self.device and (m.num_rows == 0 or m.num_cols == 0):
            x, y = np.zeros(0), np.zeros(0)
        return _result_from(res, x, y, trace)


class DeviceModel:
    """A Model whose arrays live in device memory (torch tensors on cuda)."""

    def __init__(self, model: Model, device: str = "cuda:0"):
        import torch
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.num_rows, self.num_cols, self.nnz = model.num_rows, model.num_cols, model.nnz
        self.col_start = t(model.col_start)
        self.row_index = t(model.row_index)
        self.value = t(model.value)
        self.objective = t(model.objective)
        self.var_lower = t(model.var_lower)
        self.var_upper = t(model.var_upper)
        self.row_lower = t(model.row_lower)
        self.row_upper = t(model.row_upper)
        self.objective_offset = float(model.objective_offset)
        self.objective_sense = int(model.objective_sense)

    def to_struct(self) -> _abi.McLp:
        s = _abi.McLp()
        s.num_rows, s.num_cols, s.nnz = self.num_rows, self.num_cols, self.nnz
        for k in ("col_start", "row_index", "value", "objective", "var_lower", "var_upper",
                  "row_lower", "row_upper"):
            setattr(s, k, getattr(self, k).data_ptr())
        s.objective_offset = self.objective_offset
        s.objective_sense = self.objective_sense
        s.memory = _abi.MC_MEMORY_DEVICE
        return s


_default_ctx: dict[int, Context] = {}


def solve_pdlp(model: Model, options: Optional[PdlpOptions] = None) -> PdlpResult:
    """The reference entry point (pdlp.hpp:67), on the GPU."""
    options = options or PdlpOptions()
    ctx = _default_ctx.get(options.device)
    if ctx is None:
        ctx = _default_ctx[options.device] = Context(options.device)
    return ctx.solve(model, options)
