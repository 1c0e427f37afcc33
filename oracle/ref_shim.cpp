// C shim over the reference's own CPU PDLP -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile together with the reference's sources, where
// they lie, into oracle/_ref/libref_pdlp.so.  It converts the engine's mc_lp
// (plain CSC arrays, +-INFINITY bounds) into markov_cero::model::Model and
// calls the reference entry points unchanged:
//   lp::first_order::solve_pdlp      src/lp/first_order/pdlp.cpp:139
//   scale::equilibrate_model         src/scale/ruiz_scaling.cpp:152
//   verify::verify_primal            src/verify/primal_verifier.cpp:44
//   lp::reference::solve (simplex)   src/lp/reference/revised_simplex.cpp (small LPs only)
//   io::parse_mps                    src/io/mps.cpp:96 (fixture generation)
//   presolve::presolve / postsolve   src/presolve/presolve.cpp:20, :219
// Only tests, the golden-fixture script and bench.py's reference arm use it.
#include "mc_pdlp.h"

#include "markov_cero/io/mps.hpp"
#include "markov_cero/lp/first_order/pdlp.hpp"
#include "markov_cero/lp/reference/revised_simplex.hpp"
#include "markov_cero/model/model.hpp"
#include "markov_cero/presolve/presolve.hpp"
#include "markov_cero/scale/ruiz_scaling.hpp"
#include "markov_cero/transform/sparse_canonical_model.hpp"
#include "markov_cero/verify/primal_verifier.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <string>
#include <variant>
#include <vector>

namespace mdl = markov_cero::model;
namespace fo = markov_cero::lp::first_order;

namespace {

thread_local std::string g_error;
thread_local mdl::Model g_loaded;

mdl::Bound lower_bound(double v) {
    return std::isinf(v) ? mdl::Bound::negative_infinity() : mdl::Bound::finite(v);
}
mdl::Bound upper_bound(double v) {
    return std::isinf(v) ? mdl::Bound::positive_infinity() : mdl::Bound::finite(v);
}
double from_bound(const mdl::Bound& b, double inf) {
    return b.kind == mdl::BoundKind::finite ? b.value : inf;
}

// Names are only needed by Model::validate (verify_primal); solve_pdlp never
// reads them, so large timing runs skip building millions of strings.
mdl::Model to_model(const mc_lp* lp, bool with_names = true) {
    mdl::Model model;
    model.name = "MC_LP";
    const std::size_t m = static_cast<std::size_t>(lp->num_rows);
    const std::size_t n = static_cast<std::size_t>(lp->num_cols);
    const std::size_t nnz = static_cast<std::size_t>(lp->nnz);
    model.objective_sense =
        lp->objective_sense == MC_MAXIMIZE ? mdl::ObjectiveSense::maximize : mdl::ObjectiveSense::minimize;
    model.objective_offset = lp->objective_offset;
    model.matrix.row_count = m;
    model.matrix.column_count = n;
    model.matrix.column_start.assign(lp->col_start, lp->col_start + n + 1);
    model.matrix.row_index.assign(lp->row_index, lp->row_index + nnz);
    model.matrix.value.assign(lp->value, lp->value + nnz);
    model.objective.assign(lp->objective, lp->objective + n);
    model.row_lower.resize(m);
    model.row_upper.resize(m);
    if (with_names) model.row_name.resize(m);
    for (std::size_t i = 0; i < m; ++i) {
        model.row_lower[i] = lower_bound(lp->row_lower[i]);
        model.row_upper[i] = upper_bound(lp->row_upper[i]);
        if (with_names) model.row_name[i] = "R" + std::to_string(i);
    }
    model.variable_lower.resize(n);
    model.variable_upper.resize(n);
    if (with_names) model.variable_name.resize(n);
    model.variable_type.assign(n, mdl::VariableType::continuous);
    for (std::size_t j = 0; j < n; ++j) {
        model.variable_lower[j] = lower_bound(lp->var_lower[j]);
        model.variable_upper[j] = upper_bound(lp->var_upper[j]);
        if (with_names) model.variable_name[j] = "C" + std::to_string(j);
    }
    return model;
}

fo::PdlpOptions to_options(const mc_pdlp_options* o) {
    fo::PdlpOptions p;
    p.max_iterations = static_cast<std::size_t>(o->max_iterations);
    p.restart_every = static_cast<std::size_t>(o->restart_every);
    p.primal_tolerance = o->primal_tolerance;
    p.dual_tolerance = o->dual_tolerance;
    p.gap_tolerance = o->gap_tolerance;
    p.step_size_reduction = o->step_size_reduction;
    p.power_iterations = static_cast<std::size_t>(o->power_iterations);
    p.backend = fo::Backend::cpu;
    p.restart_strategy = o->restart_strategy == MC_RESTART_NONE   ? fo::RestartStrategy::none
                         : o->restart_strategy == MC_RESTART_FIXED ? fo::RestartStrategy::fixed
                                                                   : fo::RestartStrategy::adaptive;
    p.restart_reduction_factor = o->restart_reduction_factor;
    p.adaptive_step_size = o->adaptive_step_size != 0;
    p.adaptive_primal_weight = o->adaptive_primal_weight != 0;
    p.initial_primal_weight = o->initial_primal_weight;
    p.primal_weight_smoothing = o->primal_weight_smoothing;
    p.ruiz_scaling = o->ruiz_scaling != 0;
    p.ruiz_iterations = static_cast<std::size_t>(o->ruiz_iterations);
    return p;
}

} // namespace

extern "C" {

int ref_last_error(char* buf, size_t len) {
    if (buf && len) std::snprintf(buf, len, "%s", g_error.c_str());
    return 0;
}

// The reference solve, exactly as a library caller runs it.
int ref_solve_pdlp(const mc_lp* lp, const mc_pdlp_options* o, double* primal_out,
                   double* dual_out, mc_pdlp_result* r) {
    try {
        const mdl::Model model = to_model(lp, false);
        const fo::PdlpResult res = fo::solve_pdlp(model, to_options(o));
        std::memset(r, 0, sizeof *r);
        r->status = static_cast<int32_t>(res.status);
        r->objective = res.objective;
        r->primal_infeasibility = res.primal_infeasibility;
        r->dual_infeasibility = res.dual_infeasibility;
        r->duality_gap = res.duality_gap;
        r->tolerance = res.tolerance;
        r->iterations = static_cast<int64_t>(res.iterations);
        std::snprintf(r->message, sizeof r->message, "%s", res.message.c_str());
        r->h2d_ms = res.h2d_ms;
        r->kernel_ms = res.kernel_ms;
        r->d2h_ms = res.d2h_ms;
        r->total_ms = res.total_ms;
        std::snprintf(r->backend_actually_used, sizeof r->backend_actually_used, "%s",
                      res.backend_actually_used.c_str());
        if (primal_out && !res.primal.empty())
            std::memcpy(primal_out, res.primal.data(), res.primal.size() * sizeof(double));
        if (dual_out && !res.dual.empty())
            std::memcpy(dual_out, res.dual.data(), res.dual.size() * sizeof(double));
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// equilibrate_model on the mc_lp copy; outputs the scaled arrays.
int ref_equilibrate_model(const mc_lp* lp, int64_t max_iterations, double* value,
                          double* objective, double* var_lower, double* var_upper,
                          double* row_lower, double* row_upper, double* row_scale,
                          double* col_scale, int64_t* iterations_executed, int32_t* converged) {
    try {
        mdl::Model model = to_model(lp, false);
        markov_cero::scale::RuizOptions ro;
        ro.max_iterations = static_cast<std::size_t>(max_iterations);
        const auto sc = markov_cero::scale::equilibrate_model(model, ro);
        const std::size_t m = model.matrix.row_count, n = model.matrix.column_count;
        std::memcpy(value, model.matrix.value.data(), model.matrix.value.size() * sizeof(double));
        for (std::size_t j = 0; j < n; ++j) {
            objective[j] = model.objective[j];
            var_lower[j] = from_bound(model.variable_lower[j], -INFINITY);
            var_upper[j] = from_bound(model.variable_upper[j], INFINITY);
            col_scale[j] = sc.col_scale[j];
        }
        for (std::size_t i = 0; i < m; ++i) {
            row_lower[i] = from_bound(model.row_lower[i], -INFINITY);
            row_upper[i] = from_bound(model.row_upper[i], INFINITY);
            row_scale[i] = sc.row_scale[i];
        }
        *iterations_executed = static_cast<int64_t>(sc.iterations_executed);
        *converged = sc.converged ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// verify_primal with tolerance `tol` for feasibility, objective and integrality
// (the CLI's PDLP call, apps/markov_cero_solve.cpp:164-168).
int ref_verify_primal(const mc_lp* lp, const double* primal, double claimed_objective, double tol,
                      int32_t* passed, double* max_row_violation, double* max_var_violation,
                      double* recomputed_objective) {
    try {
        const mdl::Model model = to_model(lp);
        markov_cero::verify::Candidate cand{
            std::vector<double>(primal, primal + lp->num_cols), claimed_objective};
        const markov_cero::verify::Tolerance t{tol, tol};
        const auto rep = markov_cero::verify::verify_primal(model, cand, t, t, tol);
        *passed = rep.passed ? 1 : 0;
        *max_row_violation = rep.maximum_row_violation;
        *max_var_violation = rep.maximum_variable_violation;
        *recomputed_objective = rep.recomputed_objective;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// The reference's primal simplex on a small LP, along the CLI's path without
// presolve or scaling (apps/markov_cero_solve.cpp:275-276, :311, :332,
// :393-394): sparse_canonicalize -> to_dense -> lp::reference::solve ->
// reconstruct_primal / reconstruct_objective.  The simplex keeps its own
// limits (src/lp/reference/revised_simplex.cpp:15-17, :252-257): a model past
// them returns 1 with the reference's length_error message.
// status: the reference's SolveStatus order (optimal 0, infeasible 1,
// unbounded 2, iteration_limit 3, ...).
int ref_simplex_solve(const mc_lp* lp, int64_t iteration_limit, double* primal_out,
                      double* objective_out, int32_t* status, int64_t* iterations) {
    try {
        const mdl::Model model = to_model(lp);
        const auto sparse = markov_cero::transform::sparse_canonicalize(model, /*relax_integrality=*/true);
        const auto dense = sparse.to_dense();
        markov_cero::lp::reference::Options ro;
        if (iteration_limit > 0) ro.iteration_limit = static_cast<std::size_t>(iteration_limit);
        const auto res = markov_cero::lp::reference::solve(dense, ro);
        *status = static_cast<int32_t>(res.status);
        *iterations = static_cast<int64_t>(res.phase_one_iterations + res.phase_two_iterations);
        if (res.status == markov_cero::lp::reference::SolveStatus::optimal) {
            const auto x = markov_cero::transform::reconstruct_primal(sparse, res.primal);
            if (primal_out) std::memcpy(primal_out, x.data(), x.size() * sizeof(double));
            *objective_out = markov_cero::transform::reconstruct_objective(sparse, res.objective);
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// The full verify_primal report: counts and lowest index of the violations
// per category (variable_lower, variable_upper, row_lower, row_upper,
// objective), and recomputed objective, objective difference, maximum row and
// variable violations in out4.
int ref_verify_primal_report(const mc_lp* lp, const double* primal, double claimed_objective,
                             double feas_abs, double feas_rel, double obj_abs, double obj_rel,
                             int64_t* counts, int64_t* first, double* out4, int32_t* passed) {
    static const char* kinds[5] = {"variable_lower", "variable_upper", "row_lower", "row_upper", "objective"};
    try {
        const mdl::Model model = to_model(lp);
        markov_cero::verify::Candidate cand{
            std::vector<double>(primal, primal + lp->num_cols), claimed_objective};
        const markov_cero::verify::Tolerance ft{feas_abs, feas_rel}, ot{obj_abs, obj_rel};
        const auto rep = markov_cero::verify::verify_primal(model, cand, ft, ot, 1e-6);
        for (int k = 0; k < 5; ++k) {
            counts[k] = 0;
            first[k] = -1;
        }
        for (const auto& v : rep.violations)
            for (int k = 0; k < 5; ++k)
                if (v.category == kinds[k]) {
                    counts[k] += 1;
                    if (first[k] < 0 || (int64_t)v.index < first[k]) first[k] = (int64_t)v.index;
                }
        out4[0] = rep.recomputed_objective;
        out4[1] = rep.objective_difference;
        out4[2] = rep.maximum_row_violation;
        out4[3] = rep.maximum_variable_violation;
        *passed = rep.passed ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// The canonical model of an LP (sparse_canonicalize, as the CLI's simplex
// path builds it) and the reference's equilibrate on it
// (src/scale/ruiz_scaling.cpp:20-125).  ref_canonical_sizes gives m, n, nnz;
// ref_canonical_equilibrate writes the canonical CSC and rhs/objective before
// scaling (col_start, row_index, value_in, rhs_in, obj_in) and the results.
thread_local markov_cero::transform::SparseCanonicalModel g_canonical;

int ref_canonical_sizes(const mc_lp* lp, int64_t* m, int64_t* n, int64_t* nnz) {
    try {
        g_canonical = markov_cero::transform::sparse_canonicalize(to_model(lp), /*relax_integrality=*/true);
        *m = (int64_t)g_canonical.matrix.rows;
        *n = (int64_t)g_canonical.matrix.columns;
        *nnz = (int64_t)g_canonical.matrix.values.size();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

int ref_canonical_equilibrate(int64_t max_iterations, double tolerance, double min_scale, double max_scale,
                              int32_t* col_start, int32_t* row_index, double* value_in, double* rhs_in,
                              double* obj_in, double* value_out, double* rhs_out, double* obj_out,
                              double* row_scale, double* col_scale, double* inv_row, double* inv_col,
                              int64_t* iterations, int32_t* converged) {
    try {
        auto& c = g_canonical;
        const std::size_t m = c.matrix.rows, n = c.matrix.columns, z = c.matrix.values.size();
        for (std::size_t j = 0; j <= n; ++j) col_start[j] = (int32_t)c.matrix.column_offsets[j];
        for (std::size_t p = 0; p < z; ++p) {
            row_index[p] = (int32_t)c.matrix.row_indices[p];
            value_in[p] = c.matrix.values[p];
        }
        std::memcpy(rhs_in, c.rhs.data(), m * sizeof(double));
        std::memcpy(obj_in, c.objective.data(), n * sizeof(double));
        markov_cero::scale::RuizOptions ro;
        ro.max_iterations = (std::size_t)max_iterations;
        ro.tolerance = tolerance;
        ro.min_scale = min_scale;
        ro.max_scale = max_scale;
        const auto sc = markov_cero::scale::equilibrate(c, ro);
        std::memcpy(value_out, c.matrix.values.data(), z * sizeof(double));
        std::memcpy(rhs_out, c.rhs.data(), m * sizeof(double));
        std::memcpy(obj_out, c.objective.data(), n * sizeof(double));
        std::memcpy(row_scale, sc.row_scale.data(), m * sizeof(double));
        std::memcpy(col_scale, sc.col_scale.data(), n * sizeof(double));
        std::memcpy(inv_row, sc.inv_row_scale.data(), m * sizeof(double));
        std::memcpy(inv_col, sc.inv_col_scale.data(), n * sizeof(double));
        *iterations = (int64_t)sc.iterations_executed;
        *converged = sc.converged ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// Parse an MPS file with the reference parser; sizes first, arrays by fetch.
int ref_mps_load(const char* path, int32_t* m, int32_t* n, int64_t* nnz, int32_t* sense,
                 double* offset) {
    try {
        std::ifstream in(path);
        if (!in) {
            g_error = std::string("cannot open ") + path;
            return 1;
        }
        g_loaded = markov_cero::io::parse_mps(in);
        *m = static_cast<int32_t>(g_loaded.matrix.row_count);
        *n = static_cast<int32_t>(g_loaded.matrix.column_count);
        *nnz = static_cast<int64_t>(g_loaded.matrix.value.size());
        *sense = g_loaded.objective_sense == mdl::ObjectiveSense::maximize ? MC_MAXIMIZE : MC_MINIMIZE;
        *offset = g_loaded.objective_offset;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

int ref_mps_fetch(int32_t* col_start, int32_t* row_index, double* value, double* objective,
                  double* var_lower, double* var_upper, double* row_lower, double* row_upper) {
    const auto& M = g_loaded;
    for (std::size_t j = 0; j <= M.matrix.column_count; ++j)
        col_start[j] = static_cast<int32_t>(M.matrix.column_start[j]);
    for (std::size_t p = 0; p < M.matrix.value.size(); ++p) {
        row_index[p] = static_cast<int32_t>(M.matrix.row_index[p]);
        value[p] = M.matrix.value[p];
    }
    for (std::size_t j = 0; j < M.matrix.column_count; ++j) {
        objective[j] = M.objective[j];
        var_lower[j] = from_bound(M.variable_lower[j], -INFINITY);
        var_upper[j] = from_bound(M.variable_upper[j], INFINITY);
    }
    for (std::size_t i = 0; i < M.matrix.row_count; ++i) {
        row_lower[i] = from_bound(M.row_lower[i], -INFINITY);
        row_upper[i] = from_bound(M.row_upper[i], INFINITY);
    }
    return 0;
}

// The canonical model kept by ref_canonical_sizes, unscaled.
int ref_canonical_fetch(int32_t* col_start, int32_t* row_index, double* value, double* rhs, double* obj,
                        double* offset) {
    const auto& c = g_canonical;
    for (std::size_t j = 0; j <= c.matrix.columns; ++j) col_start[j] = (int32_t)c.matrix.column_offsets[j];
    for (std::size_t p = 0; p < c.matrix.values.size(); ++p) {
        row_index[p] = (int32_t)c.matrix.row_indices[p];
        value[p] = c.matrix.values[p];
    }
    std::memcpy(rhs, c.rhs.data(), c.matrix.rows * sizeof(double));
    std::memcpy(obj, c.objective.data(), c.matrix.columns * sizeof(double));
    *offset = c.objective_offset;
    return 0;
}

// presolve() on a canonical model given as arrays (its canonicalisation
// record is the default one: objective sign +1, no structural-variable map);
// the result stays here for ref_presolve_fetch and ref_postsolve.
thread_local markov_cero::transform::SparseCanonicalModel g_pre_in;
thread_local markov_cero::presolve::PresolveResult g_pre;

int ref_presolve(const mc_canonical_lp* lp, const mc_presolve_options* o, mc_presolve_info* info) {
    namespace ps = markov_cero::presolve;
    try {
        auto& c = g_pre_in;
        c = markov_cero::transform::SparseCanonicalModel{};
        c.matrix.rows = (std::size_t)lp->num_rows;
        c.matrix.columns = (std::size_t)lp->num_cols;
        c.matrix.column_offsets.assign(lp->col_start, lp->col_start + lp->num_cols + 1);
        c.matrix.row_indices.assign(lp->row_index, lp->row_index + lp->nnz);
        c.matrix.values.assign(lp->value, lp->value + lp->nnz);
        c.rhs.assign(lp->rhs, lp->rhs + lp->num_rows);
        c.objective.assign(lp->objective, lp->objective + lp->num_cols);
        c.objective_offset = lp->objective_offset;
        c.record.objective_sign = 1.0;
        ps::PresolveOptions po;
        po.max_passes = (std::size_t)o->max_passes;
        po.feasibility_tolerance = o->feasibility_tolerance;
        po.dual_tolerance = o->dual_tolerance;
        po.pivot_tolerance = o->pivot_tolerance;
        g_pre = ps::presolve(c, po);
        std::memset(info, 0, sizeof *info);
        info->status = (int32_t)g_pre.status;
        std::snprintf(info->message, sizeof info->message, "%s", g_pre.message.c_str());
        const auto& st = g_pre.statistics;
        info->passes_executed = (int64_t)st.passes_executed;
        info->empty_rows_removed = (int64_t)st.empty_rows_removed;
        info->empty_cols_removed = (int64_t)st.empty_cols_removed;
        info->fixed_vars_removed = (int64_t)st.fixed_vars_removed;
        info->row_singletons_removed = (int64_t)st.row_singletons_removed;
        info->original_rows = (int64_t)st.original_rows;
        info->original_cols = (int64_t)st.original_cols;
        info->presolved_rows = (int64_t)st.presolved_rows;
        info->presolved_cols = (int64_t)st.presolved_cols;
        info->presolved_nnz = (int64_t)g_pre.model.matrix.values.size();
        info->objective_offset = g_pre.model.objective_offset;
        info->records = (int64_t)g_pre.stack.size();
        int64_t inc = 0;
        for (const auto& r : g_pre.stack.records())
            if (const auto* f = std::get_if<ps::FixedVariableRecord>(&r)) inc += (int64_t)f->row_indices.size();
        info->incident_entries = inc;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// The kept presolve result into arrays laid out as mc_presolve_get_model /
// _get_maps / _get_records give them.
int ref_presolve_fetch(int32_t* col_start, int32_t* row_index, double* values, double* rhs, double* objective,
                       int64_t* row_map, int64_t* col_map, int32_t* kind, int64_t* index, int64_t* variable,
                       double* value, double* value2, int64_t* incident_start, int64_t* incident_row,
                       double* incident_coefficient) {
    namespace ps = markov_cero::presolve;
    const auto& M = g_pre.model;
    const std::size_t nn = M.matrix.columns;
    if (M.matrix.column_offsets.size() == nn + 1)
        for (std::size_t j = 0; j <= nn; ++j) col_start[j] = (int32_t)M.matrix.column_offsets[j];
    else
        col_start[0] = 0;
    for (std::size_t p = 0; p < M.matrix.values.size(); ++p) {
        row_index[p] = (int32_t)M.matrix.row_indices[p];
        values[p] = M.matrix.values[p];
    }
    for (std::size_t i = 0; i < M.rhs.size(); ++i) rhs[i] = M.rhs[i];
    for (std::size_t j = 0; j < M.objective.size(); ++j) objective[j] = M.objective[j];
    const auto& rm = g_pre.stack.presolved_to_original_rows();
    const auto& cm = g_pre.stack.presolved_to_original_cols();
    for (std::size_t i = 0; i < rm.size(); ++i) row_map[i] = (int64_t)rm[i];
    for (std::size_t j = 0; j < cm.size(); ++j) col_map[j] = (int64_t)cm[j];
    int64_t t = 0, q = 0;
    incident_start[0] = 0;
    for (const auto& r : g_pre.stack.records()) {
        variable[t] = -1;
        value2[t] = 0.0;
        if (const auto* e = std::get_if<ps::EmptyRowRecord>(&r)) {
            kind[t] = MC_RECORD_EMPTY_ROW;
            index[t] = (int64_t)e->original_row_index;
            value[t] = e->rhs_value;
        } else if (const auto* c = std::get_if<ps::EmptyColumnRecord>(&r)) {
            kind[t] = MC_RECORD_EMPTY_COLUMN;
            index[t] = (int64_t)c->original_col_index;
            value[t] = c->objective_coeff;
            value2[t] = c->fixed_value;
        } else if (const auto* f = std::get_if<ps::FixedVariableRecord>(&r)) {
            kind[t] = MC_RECORD_FIXED_VARIABLE;
            index[t] = (int64_t)f->original_col_index;
            value[t] = f->fixed_value;
            value2[t] = f->objective_coeff;
            for (std::size_t k = 0; k < f->row_indices.size(); ++k, ++q) {
                incident_row[q] = (int64_t)f->row_indices[k];
                incident_coefficient[q] = f->coefficients[k];
            }
        } else if (const auto* s = std::get_if<ps::RowSingletonRecord>(&r)) {
            kind[t] = MC_RECORD_ROW_SINGLETON;
            index[t] = (int64_t)s->original_row_index;
            variable[t] = (int64_t)s->variable_index;
            value[t] = s->coefficient;
            value2[t] = s->rhs_value;
        }
        incident_start[++t] = q;
    }
    return 0;
}

// postsolve() of the kept result against the kept input model.
int ref_postsolve(const double* reduced_primal, int64_t reduced_cols, const double* reduced_dual,
                  int64_t reduced_rows, double* primal, double* dual, double* objective) {
    try {
        markov_cero::lp::reference::Result red;
        red.status = markov_cero::lp::reference::SolveStatus::optimal;
        red.primal.assign(reduced_primal, reduced_primal + reduced_cols);
        red.dual.assign(reduced_dual, reduced_dual + reduced_rows);
        const auto out = markov_cero::presolve::postsolve(g_pre.stack, red, g_pre_in);
        std::memcpy(primal, out.primal.data(), out.primal.size() * sizeof(double));
        std::memcpy(dual, out.dual.data(), out.dual.size() * sizeof(double));
        *objective = out.objective;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

} // extern "C"
