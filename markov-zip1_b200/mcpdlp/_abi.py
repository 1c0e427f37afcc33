"""ctypes mirror of include/mc_pdlp.h (the engine's C ABI).

Struct layouts here must match the header field for field; the tests check
sizes against the library's own ``sizeof`` report.
"""
from __future__ import annotations

import ctypes as C

MC_PDLP_ABI_VERSION = 1

MC_OK = 0
MC_ERR_INVALID_ARGUMENT = 1
MC_ERR_NO_DEVICE = 2
MC_ERR_OUT_OF_MEMORY = 3
MC_ERR_RESOURCE_LIMIT = 4
MC_ERR_CUDA = 5
MC_ERR_INTERNAL = 6

ERROR_NAMES = {
    MC_OK: "ok",
    MC_ERR_INVALID_ARGUMENT: "invalid_argument",
    MC_ERR_NO_DEVICE: "no_device",
    MC_ERR_OUT_OF_MEMORY: "out_of_memory",
    MC_ERR_RESOURCE_LIMIT: "resource_limit",
    MC_ERR_CUDA: "cuda_error",
    MC_ERR_INTERNAL: "internal_error",
}

MC_MEMORY_HOST = 0
MC_MEMORY_DEVICE = 1
MC_PRECISION_FP64 = 0
MC_PRECISION_FP32_REFINE = 1
MC_KERNEL_KINDS = 8
CERTIFICATE_NAMES = ("none", "crossed_bounds", "row_activity", "dual_ray")
KERNEL_KIND_NAMES = ("primal", "dual", "dual_step", "residual", "setup", "other", "-", "-")

_P_i32 = C.POINTER(C.c_int32)
_P_i64 = C.POINTER(C.c_int64)
_P_f64 = C.POINTER(C.c_double)


class McLp(C.Structure):
    _fields_ = [
        ("num_rows", C.c_int32),
        ("num_cols", C.c_int32),
        ("nnz", C.c_int64),
        ("col_start", C.c_void_p),
        ("row_index", C.c_void_p),
        ("value", C.c_void_p),
        ("objective", C.c_void_p),
        ("var_lower", C.c_void_p),
        ("var_upper", C.c_void_p),
        ("row_lower", C.c_void_p),
        ("row_upper", C.c_void_p),
        ("objective_offset", C.c_double),
        ("objective_sense", C.c_int32),
        ("memory", C.c_int32),
    ]


class McPdlpOptions(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int64),
        ("restart_every", C.c_int64),
        ("primal_tolerance", C.c_double),
        ("dual_tolerance", C.c_double),
        ("gap_tolerance", C.c_double),
        ("step_size_reduction", C.c_double),
        ("power_iterations", C.c_int64),
        ("backend", C.c_int32),
        ("restart_strategy", C.c_int32),
        ("restart_reduction_factor", C.c_double),
        ("adaptive_step_size", C.c_int32),
        ("adaptive_primal_weight", C.c_int32),
        ("initial_primal_weight", C.c_double),
        ("primal_weight_smoothing", C.c_double),
        ("ruiz_scaling", C.c_int32),
        ("ruiz_iterations", C.c_int64),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("profile_kernels", C.c_int32),
        ("check_every_chunks", C.c_int32),
        ("lanes_per_column", C.c_int32),
        ("lanes_per_row", C.c_int32),
        ("warm_start_guard", C.c_int32),
        ("reserved_i", C.c_int32 * 4),
        ("reserved_d", C.c_double * 8),
    ]


class McPdlpResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("objective", C.c_double),
        ("primal_infeasibility", C.c_double),
        ("dual_infeasibility", C.c_double),
        ("duality_gap", C.c_double),
        ("tolerance", C.c_double),
        ("iterations", C.c_int64),
        ("message", C.c_char * 160),
        ("h2d_ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("d2h_ms", C.c_double),
        ("total_ms", C.c_double),
        ("backend_actually_used", C.c_char * 16),
        ("ruiz_iterations_executed", C.c_int64),
        ("restarts", C.c_int64),
        ("final_primal_weight", C.c_double),
        ("final_step_size", C.c_double),
        ("refinement_rounds", C.c_int64),
        ("inner_iterations", C.c_int64),
        ("kernel_ms_by_kind", C.c_double * MC_KERNEL_KINDS),
        ("launches_by_kind", C.c_int64 * MC_KERNEL_KINDS),
        ("kernel_launches", C.c_int64),
        ("warm_start_used", C.c_int32),
        ("certificate", C.c_int32),
        ("warm_start_score", C.c_double),
        ("cold_start_score", C.c_double),
        ("certificate_index", C.c_int64),
        ("reserved_d1", C.c_double),
    ]


class McPdlpTrace(C.Structure):
    _fields_ = [
        ("capacity", C.c_int64),
        ("count", C.c_int64),
        ("iteration", C.c_void_p),
        ("primal_infeasibility", C.c_void_p),
        ("dual_infeasibility", C.c_void_p),
        ("duality_gap", C.c_void_p),
        ("step_size", C.c_void_p),
        ("primal_weight", C.c_void_p),
        ("restarted", C.c_void_p),
    ]


MC_VIOLATION_KINDS = 5
VIOLATION_KINDS = ("variable_lower", "variable_upper", "row_lower", "row_upper", "objective")


class McVerifyReport(C.Structure):
    _fields_ = [
        ("passed", C.c_int32),
        ("reserved0", C.c_int32),
        ("recomputed_objective", C.c_double),
        ("objective_difference", C.c_double),
        ("maximum_row_violation", C.c_double),
        ("maximum_variable_violation", C.c_double),
        ("violations", C.c_int64 * MC_VIOLATION_KINDS),
        ("first_index", C.c_int64 * MC_VIOLATION_KINDS),
        ("reserved_d", C.c_double * 4),
    ]


class McCanonicalLp(C.Structure):
    """mc_canonical_lp: SparseCanonicalModel as plain arrays."""
    _fields_ = [
        ("num_rows", C.c_int32),
        ("num_cols", C.c_int32),
        ("nnz", C.c_int64),
        ("col_start", C.c_void_p),
        ("row_index", C.c_void_p),
        ("value", C.c_void_p),
        ("rhs", C.c_void_p),
        ("objective", C.c_void_p),
        ("objective_offset", C.c_double),
    ]


class McPresolveOptions(C.Structure):
    _fields_ = [
        ("max_passes", C.c_int64),
        ("feasibility_tolerance", C.c_double),
        ("dual_tolerance", C.c_double),
        ("pivot_tolerance", C.c_double),
    ]


class McPresolveInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("message", C.c_char * 96),
        ("passes_executed", C.c_int64),
        ("empty_rows_removed", C.c_int64),
        ("empty_cols_removed", C.c_int64),
        ("fixed_vars_removed", C.c_int64),
        ("row_singletons_removed", C.c_int64),
        ("original_rows", C.c_int64),
        ("original_cols", C.c_int64),
        ("presolved_rows", C.c_int64),
        ("presolved_cols", C.c_int64),
        ("presolved_nnz", C.c_int64),
        ("objective_offset", C.c_double),
        ("records", C.c_int64),
        ("incident_entries", C.c_int64),
        ("scan_rounds", C.c_int64),
        ("presolve_ms", C.c_double),
    ]


MC_RECORD_EMPTY_ROW, MC_RECORD_EMPTY_COLUMN, MC_RECORD_FIXED_VARIABLE, MC_RECORD_ROW_SINGLETON = 0, 1, 2, 3


def default_options_struct() -> McPdlpOptions:
    """Defaults of PdlpOptions (include/markov_cero/lp/first_order/pdlp.hpp:18-41)
    plus the engine extensions; identical to mc_pdlp_default_options()."""
    o = McPdlpOptions()
    o.max_iterations = 100000
    o.restart_every = 40
    o.primal_tolerance = 1e-4
    o.dual_tolerance = 1e-4
    o.gap_tolerance = 1e-4
    o.step_size_reduction = 0.9
    o.power_iterations = 20
    o.backend = 1
    o.restart_strategy = 1
    o.restart_reduction_factor = 0.368
    o.adaptive_step_size = 1
    o.adaptive_primal_weight = 1
    o.initial_primal_weight = 0.0
    o.primal_weight_smoothing = 0.5
    o.ruiz_scaling = 1
    o.ruiz_iterations = 10
    o.precision = MC_PRECISION_FP64
    o.device = 0
    o.profile_kernels = 0
    o.check_every_chunks = 1
    return o
