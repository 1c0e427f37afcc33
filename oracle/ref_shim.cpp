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
// Only tests, the golden-fixture script and bench.py's reference arm use it.
#include "mc_pdlp.h"

#include "markov_cero/io/mps.hpp"
#include "markov_cero/lp/first_order/pdlp.hpp"
#include "markov_cero/lp/reference/revised_simplex.hpp"
#include "markov_cero/model/model.hpp"
#include "markov_cero/scale/ruiz_scaling.hpp"
#include "markov_cero/transform/sparse_canonical_model.hpp"
#include "markov_cero/verify/primal_verifier.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <string>
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

} // extern "C"
