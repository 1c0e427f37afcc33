/*
 * CPU oracle for the device presolve -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's canonical-model presolve and
 * postsolve (src/presolve/presolve.cpp:20-217 and :219-317), pinned by the
 * tests against the reference itself (compiled into oracle/_ref) and against
 * the committed golden vectors.  The reference keeps per-row and per-column
 * entry lists that it filters lazily (presolve.cpp:71-77, 95-101, 125-130);
 * an entry survives a filter while its other end is active and its value is
 * above the pivot tolerance, and nothing is ever re-activated, so counting
 * the surviving entries of the original matrix at the moment of each test
 * gives the same answers.  This file does exactly that, in the reference's
 * order, so that every floating-point operation (the right-hand-side
 * updates, presolve.cpp:155-159, and the objective offset, :162) happens in
 * the same order on the same operands.  The postsolve's long double sums
 * (presolve.cpp:284-296, :304-307) are long double here too.
 *
 * Only tests/ and bench.py's CPU-baseline leg may call this code, and only as
 * the checker.  The product never links it.
 */
#include "presolve_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t m, n;
    int64_t nnz;
    const int32_t *cs, *ri;
    const double* v;
    int32_t *rs, *ci; /* row lists in ascending column order (presolve.cpp:49-58) */
    double* rv;
} Mat;

static int build_rows(Mat* a) {
    a->rs = (int32_t*)calloc((size_t)a->m + 1, sizeof(int32_t));
    a->ci = (int32_t*)malloc(sizeof(int32_t) * (size_t)(a->nnz + 1));
    a->rv = (double*)malloc(sizeof(double) * (size_t)(a->nnz + 1));
    int32_t* cur = (int32_t*)calloc((size_t)a->m + 1, sizeof(int32_t));
    if (!a->rs || !a->ci || !a->rv || !cur) {
        free(cur);
        return -1;
    }
    for (int64_t p = 0; p < a->nnz; ++p) a->rs[a->ri[p] + 1]++;
    for (int32_t i = 0; i < a->m; ++i) a->rs[i + 1] += a->rs[i];
    for (int32_t j = 0; j < a->n; ++j)
        for (int32_t p = a->cs[j]; p < a->cs[j + 1]; ++p) {
            const int32_t r = a->ri[p];
            const int32_t q = a->rs[r] + cur[r]++;
            a->ci[q] = j;
            a->rv[q] = a->v[p];
        }
    free(cur);
    return 0;
}

static void set_msg(mc_presolve_info* info, const char* s) { snprintf(info->message, sizeof info->message, "%s", s); }

/* SparseCanonicalModel::validate (src/transform/sparse_canonicalize.cpp:20-37)
 * and SparseCsc::validate (src/linalg/sparse_basis.cpp:26-50) without the
 * 4096-row/column cap. */
static int valid(const mc_canonical_lp* lp) {
    if (lp->num_rows < 0 || lp->num_cols < 0 || lp->nnz < 0) return 0;
    if (!isfinite(lp->objective_offset)) return 0;
    if (lp->col_start[0] != 0 || lp->col_start[lp->num_cols] != lp->nnz) return 0;
    for (int32_t j = 0; j < lp->num_cols; ++j) {
        if (lp->col_start[j] > lp->col_start[j + 1]) return 0;
        for (int32_t p = lp->col_start[j]; p < lp->col_start[j + 1]; ++p) {
            if (lp->row_index[p] < 0 || lp->row_index[p] >= lp->num_rows) return 0;
            if (p > lp->col_start[j] && lp->row_index[p] <= lp->row_index[p - 1]) return 0;
            if (!isfinite(lp->value[p]) || lp->value[p] == 0.0) return 0;
        }
    }
    for (int32_t i = 0; i < lp->num_rows; ++i)
        if (!isfinite(lp->rhs[i])) return 0;
    for (int32_t j = 0; j < lp->num_cols; ++j)
        if (!isfinite(lp->objective[j])) return 0;
    return 1;
}

int oracle_presolve(const mc_canonical_lp* lp, const mc_presolve_options* o, mc_presolve_info* info,
                    oracle_presolve_out* out) {
    memset(info, 0, sizeof *info);
    if (!valid(lp)) return MC_ERR_INVALID_ARGUMENT;
    const int32_t m = lp->num_rows, n = lp->num_cols;
    const double tol = o->pivot_tolerance;
    info->status = MC_PRESOLVE_OPTIMAL;
    info->original_rows = m;
    info->original_cols = n;
    Mat a = {m, n, lp->nnz, lp->col_start, lp->row_index, lp->value, NULL, NULL, NULL};
    if (build_rows(&a)) return MC_ERR_OUT_OF_MEMORY;
    char* row_active = (char*)malloc((size_t)m + 1);
    char* col_active = (char*)malloc((size_t)n + 1);
    double* rhs = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    memset(row_active, 1, (size_t)m + 1);
    memset(col_active, 1, (size_t)n + 1);
    memcpy(rhs, lp->rhs, sizeof(double) * (size_t)m);
    double offset = lp->objective_offset;
    int64_t nrec = 0, ninc = 0;
    out->incident_start[0] = 0;
#define PUSH(K, I, V, X, X2)              \
    do {                                  \
        out->kind[nrec] = (K);            \
        out->index[nrec] = (I);           \
        out->variable[nrec] = (V);        \
        out->value[nrec] = (X);           \
        out->value2[nrec] = (X2);         \
        out->incident_start[++nrec] = ninc; \
    } while (0)

    int rc = MC_OK;
    int64_t pass = 0;
    for (; pass < o->max_passes; ++pass) {
        int64_t reductions = 0;
        /* 1. empty rows (presolve.cpp:64-88) */
        for (int32_t i = 0; i < m; ++i) {
            if (!row_active[i]) continue;
            int32_t cnt = 0;
            for (int32_t p = a.rs[i]; p < a.rs[i + 1]; ++p) cnt += col_active[a.ci[p]] && fabs(a.rv[p]) > tol;
            if (cnt == 0) {
                if (fabs(rhs[i]) > o->feasibility_tolerance) {
                    info->status = MC_PRESOLVE_INFEASIBLE;
                    set_msg(info, "presolve: empty row with non-zero RHS detected");
                    goto early;
                }
                row_active[i] = 0;
                PUSH(MC_RECORD_EMPTY_ROW, i, -1, rhs[i], 0.0);
                info->empty_rows_removed++;
                ++reductions;
            }
        }
        /* 2. empty columns (presolve.cpp:90-114) */
        for (int32_t j = 0; j < n; ++j) {
            if (!col_active[j]) continue;
            int32_t cnt = 0;
            for (int32_t p = a.cs[j]; p < a.cs[j + 1]; ++p) cnt += row_active[a.ri[p]] && fabs(a.v[p]) > tol;
            if (cnt == 0) {
                if (lp->objective[j] < -o->dual_tolerance) {
                    info->status = MC_PRESOLVE_UNBOUNDED;
                    set_msg(info, "presolve: empty column with negative cost detected");
                    goto early;
                }
                col_active[j] = 0;
                PUSH(MC_RECORD_EMPTY_COLUMN, j, -1, lp->objective[j], 0.0);
                info->empty_cols_removed++;
                ++reductions;
            }
        }
        /* 3. row singletons in row order, each fixing its variable at once
         * (presolve.cpp:119-167) */
        for (int32_t i = 0; i < m; ++i) {
            if (!row_active[i]) continue;
            int32_t cnt = 0, j = -1;
            double aij = 0.0;
            for (int32_t p = a.rs[i]; p < a.rs[i + 1]; ++p)
                if (col_active[a.ci[p]] && fabs(a.rv[p]) > tol) {
                    ++cnt;
                    j = a.ci[p];
                    aij = a.rv[p];
                }
            if (cnt != 1) continue;
            double fixed = rhs[i] / aij;
            if (fixed < -o->feasibility_tolerance) {
                info->status = MC_PRESOLVE_INFEASIBLE;
                set_msg(info, "presolve: row singleton implies negative value for canonical non-negative variable");
                goto early;
            }
            if (fixed < 0.0) fixed = 0.0;
            PUSH(MC_RECORD_ROW_SINGLETON, i, j, aij, rhs[i]);
            row_active[i] = 0;
            info->row_singletons_removed++;
            ++reductions;
            for (int32_t p = a.cs[j]; p < a.cs[j + 1]; ++p) {
                const int32_t r = a.ri[p];
                if (row_active[r] && fabs(a.v[p]) > tol) {
                    rhs[r] -= a.v[p] * fixed;
                    out->incident_row[ninc] = r;
                    out->incident_coefficient[ninc] = a.v[p];
                    ++ninc;
                }
            }
            offset += lp->objective[j] * fixed;
            PUSH(MC_RECORD_FIXED_VARIABLE, j, -1, fixed, lp->objective[j]);
            col_active[j] = 0;
            info->fixed_vars_removed++;
        }
        if (reductions == 0) break;
    }
    info->passes_executed = pass;

    /* compaction (presolve.cpp:172-214) */
    {
        int64_t nm = 0, nn = 0, nz = 0;
        int64_t* new_row = (int64_t*)malloc(sizeof(int64_t) * ((size_t)m + 1));
        for (int32_t i = 0; i < m; ++i) {
            new_row[i] = -1;
            if (row_active[i]) {
                new_row[i] = nm;
                out->row_map[nm] = i;
                out->rhs[nm] = rhs[i];
                ++nm;
            }
        }
        out->col_start[0] = 0;
        for (int32_t j = 0; j < n; ++j) {
            if (!col_active[j]) continue;
            out->col_map[nn] = j;
            out->objective[nn] = lp->objective[j];
            for (int32_t p = a.cs[j]; p < a.cs[j + 1]; ++p)
                if (row_active[a.ri[p]] && fabs(a.v[p]) > tol) {
                    out->row_index[nz] = (int32_t)new_row[a.ri[p]];
                    out->values[nz] = a.v[p];
                    ++nz;
                }
            out->col_start[++nn] = (int32_t)nz;
        }
        free(new_row);
        info->presolved_rows = nm;
        info->presolved_cols = nn;
        info->presolved_nnz = nz;
        info->objective_offset = offset;
        set_msg(info, "presolve complete");
        /* the reduced model's validate() (presolve.cpp:211-213) */
        if (nm > 0 && nn > 0) {
            for (int64_t i = 0; i < nm; ++i)
                if (!isfinite(out->rhs[i])) rc = MC_ERR_INVALID_ARGUMENT;
            if (!isfinite(offset)) rc = MC_ERR_INVALID_ARGUMENT;
        }
    }
    goto done;
early:
    /* an early return leaves the statistics' pass count at 0 and the model
     * empty (presolve.cpp:80-84, 106-110, 137-142) */
    info->presolved_rows = info->presolved_cols = info->presolved_nnz = 0;
    out->col_start[0] = 0;
done:
    info->records = nrec;
    info->incident_entries = ninc;
    free(a.rs);
    free(a.ci);
    free(a.rv);
    free(row_active);
    free(col_active);
    free(rhs);
#undef PUSH
    return rc;
}

int oracle_postsolve(const mc_canonical_lp* lp, int64_t records, const int32_t* kind, const int64_t* index,
                     const int64_t* variable, const double* value, const double* value2, int64_t presolved_rows,
                     const int64_t* row_map,
                     int64_t presolved_cols, const int64_t* col_map, const double* reduced_primal, int64_t reduced_cols,
                     const double* reduced_dual, int64_t reduced_rows, double* primal, double* dual,
                     double* objective) {
    const int32_t m = lp->num_rows, n = lp->num_cols;
    for (int32_t j = 0; j < n; ++j) primal[j] = 0.0;
    for (int32_t i = 0; i < m; ++i) dual[i] = 0.0;
    /* presolve.cpp:260-272 */
    for (int64_t q = 0; q < presolved_cols; ++q)
        if (q < reduced_cols) primal[col_map[q]] = reduced_primal[q];
    for (int64_t q = 0; q < presolved_rows; ++q)
        if (q < reduced_rows) dual[row_map[q]] = reduced_dual[q];
    /* LIFO over the records (presolve.cpp:274-301) */
    for (int64_t t = records - 1; t >= 0; --t) {
        switch (kind[t]) {
            case MC_RECORD_EMPTY_ROW: dual[index[t]] = 0.0; break;
            case MC_RECORD_EMPTY_COLUMN: primal[index[t]] = value2[t]; break; /* fixed_value */
            case MC_RECORD_FIXED_VARIABLE: primal[index[t]] = value[t]; break;
            case MC_RECORD_ROW_SINGLETON: {
                const int64_t i = index[t], k = variable[t];
                long double sum_other = 0.0L;
                for (int32_t p = lp->col_start[k]; p < lp->col_start[k + 1]; ++p)
                    if (lp->row_index[p] != i)
                        sum_other += (long double)lp->value[p] * dual[lp->row_index[p]];
                const double pi = (double)((lp->objective[k] - sum_other) / value[t]);
                if (!isfinite(pi)) return MC_ERR_INVALID_ARGUMENT;
                dual[i] = pi;
                break;
            }
            default: return MC_ERR_INVALID_ARGUMENT;
        }
    }
    /* presolve.cpp:303-308 */
    long double obj = lp->objective_offset;
    for (int32_t j = 0; j < n; ++j) obj += (long double)lp->objective[j] * primal[j];
    *objective = (double)obj;
    if (!isfinite(*objective)) return MC_ERR_INVALID_ARGUMENT;
    return MC_OK;
}
