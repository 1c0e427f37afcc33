// presolve() / postsolve() of markov-cero on the B200 engine; see
// presolve_gpu.hpp.  The canonical CSC uses size_t offsets and indices
// (linalg::SparseCsc); the engine takes int32 CSC arrays (mc_canonical_lp).
// The record stack converts one to one: mc_record_kind follows the order of
// the ReductionRecord variant (presolve_stack.hpp:38-39).
#include "presolve_gpu.hpp"

#include "mc_pdlp.h"

#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

namespace markov_cero::presolve {

namespace {

[[noreturn]] void fail(int code, const char* what) {
    char msg[512];
    mc_last_error(msg, sizeof msg);
    const std::string text = std::string(what) + ": " + msg;
    if (code == MC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(text);
    if (code == MC_ERR_RESOURCE_LIMIT) throw std::length_error(text);
    throw std::runtime_error(text);
}

int32_t to_int32(std::size_t v) {
    if (v > static_cast<std::size_t>(std::numeric_limits<int32_t>::max()))
        throw std::length_error("GPU presolve: index beyond the engine's int32 range");
    return static_cast<int32_t>(v);
}

// one engine context per host thread, created on first use
struct ThreadContext {
    mc_pdlp_ctx* ctx = nullptr;
    ~ThreadContext() {
        if (ctx) mc_pdlp_ctx_destroy(ctx);
    }
    mc_pdlp_ctx* get() {
        if (!ctx) {
            const int rc = mc_pdlp_ctx_create(0, &ctx);
            if (rc != MC_OK) {
                ctx = nullptr;
                fail(rc, "GPU presolve (no CPU fallback)");
            }
        }
        return ctx;
    }
};
thread_local ThreadContext g_ctx;

// the int32 copy of a canonical model's CSC, and the engine's view of it
struct Canonical {
    std::vector<int32_t> cs, ri;
    mc_canonical_lp lp{};
    explicit Canonical(const transform::SparseCanonicalModel& c) {
        const auto& A = c.matrix;
        cs.resize(A.column_offsets.size());
        for (std::size_t j = 0; j < cs.size(); ++j) cs[j] = to_int32(A.column_offsets[j]);
        ri.resize(A.row_indices.size());
        for (std::size_t p = 0; p < ri.size(); ++p) ri[p] = to_int32(A.row_indices[p]);
        if (cs.empty()) cs.push_back(0);
        lp.num_rows = to_int32(A.rows);
        lp.num_cols = to_int32(A.columns);
        lp.nnz = static_cast<int64_t>(A.values.size());
        lp.col_start = cs.data();
        lp.row_index = ri.data();
        lp.value = A.values.data();
        lp.rhs = c.rhs.data();
        lp.objective = c.objective.data();
        lp.objective_offset = c.objective_offset;
    }
};

struct Handle {
    mc_presolve* p = nullptr;
    ~Handle() {
        if (p) mc_presolve_free(p);
    }
};

}  // namespace

PresolveResult presolve_gpu(const transform::SparseCanonicalModel& input, const PresolveOptions& options) {
    input.validate();  // the reference's checks and exceptions (presolve.cpp:22)
    const Canonical in(input);
    mc_presolve_options o;
    o.max_passes = static_cast<int64_t>(options.max_passes);
    o.feasibility_tolerance = options.feasibility_tolerance;
    o.dual_tolerance = options.dual_tolerance;
    o.pivot_tolerance = options.pivot_tolerance;
    Handle h;
    int rc = mc_presolve_run(g_ctx.get(), &in.lp, &o, &h.p);
    if (rc != MC_OK) fail(rc, "GPU presolve");
    mc_presolve_info info;
    mc_presolve_get_info(h.p, &info);

    PresolveResult result;
    result.status = static_cast<lp::reference::SolveStatus>(info.status);
    result.message = info.message;
    auto& st = result.statistics;
    st.passes_executed = static_cast<std::size_t>(info.passes_executed);
    st.empty_rows_removed = static_cast<std::size_t>(info.empty_rows_removed);
    st.empty_cols_removed = static_cast<std::size_t>(info.empty_cols_removed);
    st.fixed_vars_removed = static_cast<std::size_t>(info.fixed_vars_removed);
    st.row_singletons_removed = static_cast<std::size_t>(info.row_singletons_removed);
    st.original_rows = static_cast<std::size_t>(info.original_rows);
    st.original_cols = static_cast<std::size_t>(info.original_cols);
    st.presolved_rows = static_cast<std::size_t>(info.presolved_rows);
    st.presolved_cols = static_cast<std::size_t>(info.presolved_cols);

    // the record stack, oldest first
    const std::size_t nr = static_cast<std::size_t>(info.records), ni = static_cast<std::size_t>(info.incident_entries);
    std::vector<int32_t> kind(nr);
    std::vector<int64_t> index(nr), variable(nr), inc_start(nr + 1), inc_row(ni);
    std::vector<double> value(nr), value2(nr), inc_coef(ni);
    rc = mc_presolve_get_records(h.p, kind.data(), index.data(), variable.data(), value.data(), value2.data(),
                                 inc_start.data(), inc_row.data(), inc_coef.data());
    if (rc != MC_OK) fail(rc, "GPU presolve records");
    for (std::size_t t = 0; t < nr; ++t) {
        const auto i = static_cast<std::size_t>(index[t]);
        switch (kind[t]) {
            case MC_RECORD_EMPTY_ROW: result.stack.push(EmptyRowRecord{i, value[t]}); break;
            case MC_RECORD_EMPTY_COLUMN: result.stack.push(EmptyColumnRecord{i, value[t], value2[t]}); break;
            case MC_RECORD_FIXED_VARIABLE: {
                FixedVariableRecord f{i, value[t], value2[t], {}, {}};
                for (int64_t q = inc_start[t]; q < inc_start[t + 1]; ++q) {
                    f.row_indices.push_back(static_cast<std::size_t>(inc_row[static_cast<std::size_t>(q)]));
                    f.coefficients.push_back(inc_coef[static_cast<std::size_t>(q)]);
                }
                result.stack.push(std::move(f));
                break;
            }
            default:
                result.stack.push(RowSingletonRecord{i, static_cast<std::size_t>(variable[t]), value[t], value2[t]});
        }
    }
    if (result.status != lp::reference::SolveStatus::optimal) return result;  // default model, as the reference

    const std::size_t nm = static_cast<std::size_t>(info.presolved_rows), nc = static_cast<std::size_t>(info.presolved_cols);
    const std::size_t nz = static_cast<std::size_t>(info.presolved_nnz);
    std::vector<int64_t> rmap(nm), cmap(nc);
    rc = mc_presolve_get_maps(h.p, rmap.data(), cmap.data());
    if (rc != MC_OK) fail(rc, "GPU presolve maps");
    result.stack.set_row_map(std::vector<std::size_t>(rmap.begin(), rmap.end()));
    result.stack.set_col_map(std::vector<std::size_t>(cmap.begin(), cmap.end()));
    std::vector<int32_t> cs(nc + 1), ri(nz);
    auto& M = result.model;
    M.matrix.rows = nm;
    M.matrix.columns = nc;
    M.matrix.values.resize(nz);
    M.rhs.resize(nm);
    M.objective.resize(nc);
    rc = mc_presolve_get_model(h.p, cs.data(), ri.data(), M.matrix.values.data(), M.rhs.data(), M.objective.data());
    if (rc != MC_OK) fail(rc, "GPU presolve model");
    M.matrix.column_offsets.assign(cs.begin(), cs.end());
    M.matrix.row_indices.assign(ri.begin(), ri.end());
    M.objective_offset = info.objective_offset;
    M.record = input.record;
    if (nm > 0 && nc > 0) M.validate();  // presolve.cpp:211-213
    return result;
}

lp::reference::Result postsolve_gpu(const PresolveStack& stack, const lp::reference::Result& reduced_solution,
                                    const transform::SparseCanonicalModel& original_model, double /*tolerance*/) {
    const Canonical in(original_model);
    const auto& recs = stack.records();
    const std::size_t nr = recs.size();
    std::vector<int32_t> kind(nr);
    std::vector<int64_t> index(nr), variable(nr, -1);
    std::vector<double> value(nr), value2(nr, 0.0);
    for (std::size_t t = 0; t < nr; ++t) {
        std::visit(
            [&](const auto& r) {
                using T = std::decay_t<decltype(r)>;
                if constexpr (std::is_same_v<T, EmptyRowRecord>) {
                    kind[t] = MC_RECORD_EMPTY_ROW;
                    index[t] = static_cast<int64_t>(r.original_row_index);
                    value[t] = r.rhs_value;
                } else if constexpr (std::is_same_v<T, EmptyColumnRecord>) {
                    kind[t] = MC_RECORD_EMPTY_COLUMN;
                    index[t] = static_cast<int64_t>(r.original_col_index);
                    value[t] = r.objective_coeff;
                    value2[t] = r.fixed_value;
                } else if constexpr (std::is_same_v<T, FixedVariableRecord>) {
                    kind[t] = MC_RECORD_FIXED_VARIABLE;
                    index[t] = static_cast<int64_t>(r.original_col_index);
                    value[t] = r.fixed_value;
                    value2[t] = r.objective_coeff;
                } else {
                    kind[t] = MC_RECORD_ROW_SINGLETON;
                    index[t] = static_cast<int64_t>(r.original_row_index);
                    variable[t] = static_cast<int64_t>(r.variable_index);
                    value[t] = r.coefficient;
                    value2[t] = r.rhs_value;
                }
            },
            recs[t]);
    }
    const auto& rm = stack.presolved_to_original_rows();
    const auto& cm = stack.presolved_to_original_cols();
    std::vector<int64_t> rmap(rm.begin(), rm.end()), cmap(cm.begin(), cm.end());
    Handle h;
    mc_pdlp_ctx* ctx = g_ctx.get();
    int rc = mc_presolve_load(ctx, &in.lp, static_cast<int64_t>(nr), kind.data(), index.data(), variable.data(),
                              value.data(), value2.data(), static_cast<int64_t>(rmap.size()), rmap.data(),
                              static_cast<int64_t>(cmap.size()), cmap.data(), &h.p);
    if (rc != MC_OK) fail(rc, "GPU postsolve");
    lp::reference::Result restored = reduced_solution;
    restored.primal.assign(original_model.matrix.columns, 0.0);
    restored.dual.assign(original_model.matrix.rows, 0.0);
    double objective = 0.0;
    rc = mc_postsolve(ctx, h.p, reduced_solution.primal.data(), static_cast<int64_t>(reduced_solution.primal.size()),
                      reduced_solution.dual.data(), static_cast<int64_t>(reduced_solution.dual.size()),
                      restored.primal.data(), restored.dual.data(), &objective);
    if (rc == MC_ERR_INVALID_ARGUMENT) {
        char msg[512];
        mc_last_error(msg, sizeof msg);
        throw std::overflow_error(msg);  // presolve.cpp:297-298, :307
    }
    if (rc != MC_OK) fail(rc, "GPU postsolve");
    restored.objective = objective;
    return restored;
}

}  // namespace markov_cero::presolve
