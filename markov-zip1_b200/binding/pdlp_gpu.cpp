// solve_pdlp on the B200 engine for markov-cero's Backend::gpu.
//
// Model conversion: the reference's CSC uses size_t pointers and indices and
// a Bound{kind, value} per bound (model.hpp:15-34); the engine takes int32
// CSC arrays and +-INFINITY for infinite bounds (mc_lp, include/mc_pdlp.h).
// Options map field by field onto mc_pdlp_options; the result fills every
// PdlpResult field the CPU path fills (pdlp.cpp:263-276), with the unscaled
// averages as primal/dual.
#include "pdlp_gpu.hpp"

#include "mc_pdlp.h"

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace markov_cero::gpu {

namespace {

using lp::first_order::Backend;
using lp::first_order::PdlpOptions;
using lp::first_order::PdlpResult;
using lp::first_order::PdlpStatus;

double lower_value(const model::Bound& b) {
    if (b.kind == model::BoundKind::finite) return b.value;
    return b.kind == model::BoundKind::negative_infinity ? -INFINITY : INFINITY;
}
double upper_value(const model::Bound& b) {
    if (b.kind == model::BoundKind::finite) return b.value;
    return b.kind == model::BoundKind::positive_infinity ? INFINITY : -INFINITY;
}

[[noreturn]] void throw_engine_error(int code) {
    char msg[512];
    mc_last_error(msg, sizeof msg);
    const std::string text = std::string("GPU PDLP: ") + msg;
    if (code == MC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(text);
    if (code == MC_ERR_RESOURCE_LIMIT) throw std::length_error(text);
    throw std::runtime_error(text);
}

int32_t checked_int32(std::size_t v, const char* what) {
    if (v > static_cast<std::size_t>(std::numeric_limits<int32_t>::max()))
        throw std::length_error(std::string("GPU PDLP: ") + what + " beyond the engine's int32 range");
    return static_cast<int32_t>(v);
}

}  // namespace

bool gpu_requested(const PdlpOptions& options) {
    if (options.backend == Backend::gpu) return true;
    const char* env = std::getenv("MARKOV_CERO_PDLP_BACKEND");
    return env != nullptr && std::strcmp(env, "gpu") == 0;
}

PdlpResult solve_pdlp_gpu(const model::Model& model, const PdlpOptions& options) {
    const model::SparseMatrixCSC& A = model.matrix;
    const std::size_t m = A.row_count, n = A.column_count, nnz = A.value.size();
    if (A.column_start.size() != n + 1 || A.row_index.size() != nnz || model.objective.size() != n ||
        model.variable_lower.size() != n || model.variable_upper.size() != n ||
        model.row_lower.size() != m || model.row_upper.size() != m)
        throw std::invalid_argument("GPU PDLP: model arrays do not match the matrix dimensions");

    std::vector<int32_t> col_start(n + 1), row_index(nnz);
    for (std::size_t j = 0; j <= n; ++j) col_start[j] = checked_int32(A.column_start[j], "nonzero count");
    for (std::size_t p = 0; p < nnz; ++p) row_index[p] = checked_int32(A.row_index[p], "row index");
    std::vector<double> vl(n), vu(n), rl(m), ru(m);
    for (std::size_t j = 0; j < n; ++j) {
        vl[j] = lower_value(model.variable_lower[j]);
        vu[j] = upper_value(model.variable_upper[j]);
    }
    for (std::size_t i = 0; i < m; ++i) {
        rl[i] = lower_value(model.row_lower[i]);
        ru[i] = upper_value(model.row_upper[i]);
    }

    mc_lp lp{};
    lp.num_rows = checked_int32(m, "row count");
    lp.num_cols = checked_int32(n, "column count");
    lp.nnz = static_cast<int64_t>(nnz);
    lp.col_start = col_start.data();
    lp.row_index = row_index.data();
    lp.value = A.value.data();
    lp.objective = model.objective.data();
    lp.var_lower = vl.data();
    lp.var_upper = vu.data();
    lp.row_lower = rl.data();
    lp.row_upper = ru.data();
    lp.objective_offset = model.objective_offset;
    lp.objective_sense = model.objective_sense == model::ObjectiveSense::maximize ? MC_MAXIMIZE : MC_MINIMIZE;
    lp.memory = MC_MEMORY_HOST;

    mc_pdlp_options o;
    mc_pdlp_default_options(&o);
    o.max_iterations = static_cast<int64_t>(options.max_iterations);
    o.restart_every = static_cast<int64_t>(options.restart_every);
    o.primal_tolerance = options.primal_tolerance;
    o.dual_tolerance = options.dual_tolerance;
    o.gap_tolerance = options.gap_tolerance;
    o.step_size_reduction = options.step_size_reduction;
    o.power_iterations = static_cast<int64_t>(options.power_iterations);
    o.backend = MC_BACKEND_GPU;
    o.restart_strategy = static_cast<int32_t>(options.restart_strategy);
    o.restart_reduction_factor = options.restart_reduction_factor;
    o.adaptive_step_size = options.adaptive_step_size ? 1 : 0;
    o.adaptive_primal_weight = options.adaptive_primal_weight ? 1 : 0;
    o.initial_primal_weight = options.initial_primal_weight;
    o.primal_weight_smoothing = options.primal_weight_smoothing;
    o.ruiz_scaling = options.ruiz_scaling ? 1 : 0;
    o.ruiz_iterations = static_cast<int64_t>(options.ruiz_iterations);

    PdlpResult res;
    res.primal.assign(n, 0.0);
    res.dual.assign(m, 0.0);
    mc_pdlp_result r;
    const int rc = mc_pdlp_solve(&lp, &o, nullptr, nullptr, res.primal.data(), res.dual.data(), &r);
    if (rc != MC_OK) throw_engine_error(rc);
    res.status = static_cast<PdlpStatus>(r.status);
    res.objective = r.objective;
    res.primal_infeasibility = r.primal_infeasibility;
    res.dual_infeasibility = r.dual_infeasibility;
    res.duality_gap = r.duality_gap;
    res.tolerance = r.tolerance;
    res.iterations = static_cast<std::size_t>(r.iterations);
    res.message = r.message;
    res.h2d_ms = r.h2d_ms;
    res.kernel_ms = r.kernel_ms;
    res.d2h_ms = r.d2h_ms;
    res.total_ms = r.total_ms;
    res.backend_actually_used = r.backend_actually_used;  // "cuda"
    if (m == 0 || n == 0) {  // the trivial result carries no vectors (pdlp.cpp:144-148)
        res.primal.clear();
        res.dual.clear();
    }
    return res;
}

}  // namespace markov_cero::gpu
