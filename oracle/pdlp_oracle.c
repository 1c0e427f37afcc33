/*
 * CPU oracle for the PDLP engine -- TEST INFRASTRUCTURE ONLY (see
 * pdlp_oracle.h).  Each function names the reference lines it restates.
 * Build with -ffp-contract=off so no multiply-add is fused: the reference is
 * built for plain x86-64 and never fuses either.
 */
#include "pdlp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define BIG 1e300

/* std::clamp(v, lo, hi) */
static inline double clampd(double v, double lo, double hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}
/* std::max / std::min (first argument wins ties) */
static inline double maxd(double a, double b) { return (a < b) ? b : a; }
static inline double mind(double a, double b) { return (b < a) ? b : a; }

static double now_ms(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
}

/* BoundKind sentinels of the reference: -1e300 / +1e300 for infinite bounds
 * (pdlp.cpp:47-48, :83-84, :163-164). */
static inline double lo_sentinel(double v) { return isinf(v) ? -BIG : v; }
static inline double hi_sentinel(double v) { return isinf(v) ? BIG : v; }

/* equilibrate_model, src/scale/ruiz_scaling.cpp:152-247.  Bounds are in the
 * +-INFINITY encoding: only finite ones are scaled (:229-243). */
int oracle_equilibrate(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                       double* value, double* objective, double* var_lower, double* var_upper,
                       double* row_lower, double* row_upper, int64_t max_iterations,
                       double tolerance, double* row_scale, double* col_scale,
                       int64_t* iterations_executed, int32_t* converged) {
    for (int32_t i = 0; i < m; ++i) row_scale[i] = 1.0;
    for (int32_t j = 0; j < n; ++j) col_scale[j] = 1.0;
    *iterations_executed = 0;
    *converged = 0;
    const int64_t nnz = (n > 0) ? col_start[n] : 0;
    if (m == 0 || n == 0 || nnz == 0) return 0; /* :162-164 */

    double* r_norm = (double*)malloc(sizeof(double) * (size_t)m);
    double* c_norm = (double*)malloc(sizeof(double) * (size_t)n);
    double* delta_r = (double*)malloc(sizeof(double) * (size_t)m);
    double* delta_c = (double*)malloc(sizeof(double) * (size_t)n);
    if (!r_norm || !c_norm || !delta_r || !delta_c) {
        free(r_norm); free(c_norm); free(delta_r); free(delta_c);
        return -1;
    }
    int64_t iter = 0;
    for (; iter < max_iterations; ++iter) {                     /* :167 */
        for (int32_t i = 0; i < m; ++i) r_norm[i] = 0.0;
        for (int32_t j = 0; j < n; ++j) c_norm[j] = 0.0;
        for (int32_t col = 0; col < n; ++col) {                 /* :170-177 */
            for (int32_t p = col_start[col]; p < col_start[col + 1]; ++p) {
                const double v = fabs(value[p]);
                c_norm[col] = maxd(c_norm[col], v);
                r_norm[row_index[p]] = maxd(r_norm[row_index[p]], v);
            }
        }
        for (int32_t i = 0; i < m; ++i) if (r_norm[i] == 0.0) r_norm[i] = 1.0; /* :178-183 */
        for (int32_t j = 0; j < n; ++j) if (c_norm[j] == 0.0) c_norm[j] = 1.0;
        double max_r_err = 0.0, max_c_err = 0.0;                /* :185-192 */
        for (int32_t i = 0; i < m; ++i) max_r_err = maxd(max_r_err, fabs(1.0 - r_norm[i]));
        for (int32_t j = 0; j < n; ++j) max_c_err = maxd(max_c_err, fabs(1.0 - c_norm[j]));
        if (max_r_err < tolerance && max_c_err < tolerance) {   /* :194-197 */
            *converged = 1;
            break;
        }
        for (int32_t i = 0; i < m; ++i) {                       /* :199-208 */
            delta_r[i] = 1.0 / sqrt(r_norm[i]);
            row_scale[i] *= delta_r[i];
        }
        for (int32_t j = 0; j < n; ++j) {
            delta_c[j] = 1.0 / sqrt(c_norm[j]);
            col_scale[j] *= delta_c[j];
        }
        for (int32_t col = 0; col < n; ++col) {                 /* :210-217 */
            const double dc = delta_c[col];
            for (int32_t p = col_start[col]; p < col_start[col + 1]; ++p)
                value[p] *= delta_r[row_index[p]] * dc;
        }
    }
    *iterations_executed = iter;                                 /* :219 */
    /* :221-244: inv scales, then bounds and objective */
    for (int32_t i = 0; i < m; ++i) {
        const double s = row_scale[i];
        if (isfinite(row_lower[i])) row_lower[i] *= s;
        if (isfinite(row_upper[i])) row_upper[i] *= s;
    }
    for (int32_t j = 0; j < n; ++j) {
        const double inv = 1.0 / col_scale[j];
        if (isfinite(var_lower[j])) var_lower[j] *= inv;
        if (isfinite(var_upper[j])) var_upper[j] *= inv;
        objective[j] *= col_scale[j];
    }
    free(r_norm); free(c_norm); free(delta_r); free(delta_c);
    return 0;
}

/* spmv, pdlp.cpp:22-32 */
void oracle_spmv(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                 const double* value, const double* x, double* y) {
    for (int32_t i = 0; i < m; ++i) y[i] = 0.0;
    for (int32_t col = 0; col < n; ++col) {
        const double xc = x[col];
        if (xc == 0.0) continue;
        for (int32_t p = col_start[col]; p < col_start[col + 1]; ++p)
            y[row_index[p]] += value[p] * xc;
    }
}

/* spmv_t, pdlp.cpp:34-44 */
void oracle_spmv_t(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                   const double* value, const double* y, double* z) {
    (void)m;
    for (int32_t col = 0; col < n; ++col) {
        double s = 0.0;
        for (int32_t p = col_start[col]; p < col_start[col + 1]; ++p)
            s += value[p] * y[row_index[p]];
        z[col] = s;
    }
}

typedef struct {
    double primal_infeas, dual_infeas, duality_gap, score, objective;
} residuals_t;

/* compute_unscaled_residuals, pdlp.cpp:62-135.  `lp` is the ORIGINAL model;
 * x_out/y_out receive the unscaled averages (:74-79). */
static residuals_t unscaled_residuals(const mc_lp* lp, const double* x_avg, const double* y_avg,
                                      const double* Ax_avg, const double* At_y_avg,
                                      const double* row_scale, const double* col_scale,
                                      int ruiz, double* xu, double* yu) {
    const int32_t m = lp->num_rows, n = lp->num_cols;
    const double obj_sign = (lp->objective_sense == MC_MAXIMIZE) ? -1.0 : 1.0;
    residuals_t res;
    for (int32_t j = 0; j < n; ++j) xu[j] = ruiz ? (x_avg[j] * col_scale[j]) : x_avg[j];
    for (int32_t i = 0; i < m; ++i) yu[i] = ruiz ? (y_avg[i] * row_scale[i]) : y_avg[i];
    double max_prim_viol = 0.0;
    for (int32_t i = 0; i < m; ++i) {                                       /* :81-89 */
        const double ax_i = ruiz ? (Ax_avg[i] / row_scale[i]) : Ax_avg[i];
        const double lo = lo_sentinel(lp->row_lower[i]);
        const double hi = hi_sentinel(lp->row_upper[i]);
        const double proj = clampd(ax_i, lo, hi);
        const double r = fabs(ax_i - proj);
        const double scale = 1.0 + maxd(fabs(ax_i), fabs(proj) < 1e299 ? fabs(proj) : 0.0);
        max_prim_viol = maxd(max_prim_viol, r / scale);
    }
    for (int32_t j = 0; j < n; ++j) {                                       /* :90-97 */
        const double lo = lo_sentinel(lp->var_lower[j]);
        const double hi = hi_sentinel(lp->var_upper[j]);
        const double proj = clampd(xu[j], lo, hi);
        const double r = fabs(xu[j] - proj);
        const double scale = 1.0 + maxd(fabs(xu[j]), fabs(proj) < 1e299 ? fabs(proj) : 0.0);
        max_prim_viol = maxd(max_prim_viol, r / scale);
    }
    res.primal_infeas = max_prim_viol;
    double c_scale = 1.0, dual_res_sq = 0.0;                                /* :99-112 */
    for (int32_t j = 0; j < n; ++j) {
        const double at_y = ruiz ? (At_y_avg[j] / col_scale[j]) : At_y_avg[j];
        const double c_orig = obj_sign * lp->objective[j];
        c_scale = maxd(c_scale, fabs(c_orig));
        const double g = c_orig + at_y;
        const double lo = lo_sentinel(lp->var_lower[j]);
        const double hi = hi_sentinel(lp->var_upper[j]);
        const double x_proj = clampd(xu[j] - g, lo, hi);
        const double diff = xu[j] - x_proj;
        dual_res_sq += diff * diff;
    }
    res.dual_infeas = sqrt(dual_res_sq) / c_scale;
    double primal_obj = lp->objective_offset;                               /* :113-115 */
    for (int32_t j = 0; j < n; ++j) primal_obj += lp->objective[j] * xu[j];
    res.objective = primal_obj;
    double dual_obj = lp->objective_offset;                                 /* :116-131 */
    for (int32_t i = 0; i < m; ++i) {
        const double lo = lo_sentinel(lp->row_lower[i]);
        const double hi = hi_sentinel(lp->row_upper[i]);
        if (yu[i] > 0.0 && hi < 1e299) dual_obj -= yu[i] * hi;
        else if (yu[i] < 0.0 && lo > -1e299) dual_obj -= yu[i] * lo;
    }
    for (int32_t j = 0; j < n; ++j) {
        const double at_y = ruiz ? (At_y_avg[j] / col_scale[j]) : At_y_avg[j];
        const double c_orig = obj_sign * lp->objective[j];
        const double g = c_orig + at_y;
        const double lo = lo_sentinel(lp->var_lower[j]);
        const double hi = hi_sentinel(lp->var_upper[j]);
        if (g > 0.0 && lo > -1e299) dual_obj += g * lo;
        else if (g < 0.0 && hi < 1e299) dual_obj += g * hi;
    }
    res.duality_gap = fabs(primal_obj - dual_obj) / (1.0 + fabs(primal_obj) + fabs(dual_obj));
    res.score = maxd(maxd(res.primal_infeas, res.dual_infeas), res.duality_gap); /* :133 */
    return res;
}

static void set_message(mc_pdlp_result* r, const char* msg) {
    snprintf(r->message, sizeof r->message, "%s", msg);
}

/* solve_pdlp, pdlp.cpp:139-276 (plus the warm start extension). */
int oracle_solve_pdlp(const mc_lp* lp, const mc_pdlp_options* o,
                      const double* initial_primal, const double* initial_dual,
                      double* primal_out, double* dual_out, mc_pdlp_result* result,
                      mc_pdlp_trace* trace) {
    const double t_start = now_ms();
    memset(result, 0, sizeof *result);
    snprintf(result->backend_actually_used, sizeof result->backend_actually_used, "cpu");
    if (trace) trace->count = 0;
    if (!lp || !o || lp->num_rows < 0 || lp->num_cols < 0) return MC_ERR_INVALID_ARGUMENT;
    const int32_t m = lp->num_rows, n = lp->num_cols;
    if (n == 0 || m == 0) {                                                 /* :144-149 */
        result->status = MC_PDLP_OPTIMAL;
        result->tolerance = o->primal_tolerance;
        set_message(result, "trivial");
        return MC_OK;
    }
    const int64_t nnz = lp->col_start[n];
    /* model copy (:150) */
    double* val = (double*)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    double* obj = (double*)malloc(sizeof(double) * (size_t)n);
    double* vlo = (double*)malloc(sizeof(double) * (size_t)n);
    double* vhi = (double*)malloc(sizeof(double) * (size_t)n);
    double* rlo = (double*)malloc(sizeof(double) * (size_t)m);
    double* rhi = (double*)malloc(sizeof(double) * (size_t)m);
    double* row_scale = (double*)malloc(sizeof(double) * (size_t)m);
    double* col_scale = (double*)malloc(sizeof(double) * (size_t)n);
    double* c = (double*)malloc(sizeof(double) * (size_t)n);
    double* b_lo = (double*)malloc(sizeof(double) * (size_t)m);
    double* b_hi = (double*)malloc(sizeof(double) * (size_t)m);
    double* row_norms = (double*)calloc((size_t)m, sizeof(double));
    double* col_norms = (double*)calloc((size_t)n, sizeof(double));
    double* tau = (double*)malloc(sizeof(double) * (size_t)n);
    double* sigma = (double*)malloc(sizeof(double) * (size_t)m);
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* x_prev = (double*)malloc(sizeof(double) * (size_t)n);
    double* x_bar = (double*)malloc(sizeof(double) * (size_t)n);
    double* x_avg = (double*)malloc(sizeof(double) * (size_t)n);
    double* delta_x = (double*)calloc((size_t)n, sizeof(double));
    double* y = (double*)calloc((size_t)m, sizeof(double));
    double* y_avg = (double*)calloc((size_t)m, sizeof(double));
    double* At_y = (double*)malloc(sizeof(double) * (size_t)n);
    double* Ax = (double*)malloc(sizeof(double) * (size_t)m);
    double* xu = (double*)malloc(sizeof(double) * (size_t)n);
    double* yu = (double*)malloc(sizeof(double) * (size_t)m);
    int rc = MC_OK;
    if (!val || !obj || !vlo || !vhi || !rlo || !rhi || !row_scale || !col_scale || !c || !b_lo ||
        !b_hi || !row_norms || !col_norms || !tau || !sigma || !x || !x_prev || !x_bar || !x_avg ||
        !delta_x || !y || !y_avg || !At_y || !Ax || !xu || !yu) {
        rc = MC_ERR_OUT_OF_MEMORY;
        goto done;
    }
    memcpy(val, lp->value, sizeof(double) * (size_t)nnz);
    memcpy(obj, lp->objective, sizeof(double) * (size_t)n);
    memcpy(vlo, lp->var_lower, sizeof(double) * (size_t)n);
    memcpy(vhi, lp->var_upper, sizeof(double) * (size_t)n);
    memcpy(rlo, lp->row_lower, sizeof(double) * (size_t)m);
    memcpy(rhi, lp->row_upper, sizeof(double) * (size_t)m);
    for (int32_t i = 0; i < m; ++i) row_scale[i] = 1.0;
    for (int32_t j = 0; j < n; ++j) col_scale[j] = 1.0;
    const int ruiz = o->ruiz_scaling != 0;
    if (ruiz) {                                                             /* :151-152 */
        int32_t conv = 0;
        int64_t it = 0;
        if (oracle_equilibrate(m, n, lp->col_start, lp->row_index, val, obj, vlo, vhi, rlo, rhi,
                               o->ruiz_iterations, 1e-3, row_scale, col_scale, &it, &conv) != 0) {
            rc = MC_ERR_OUT_OF_MEMORY;
            goto done;
        }
        result->ruiz_iterations_executed = it;
    }
    const double obj_sign = (lp->objective_sense == MC_MAXIMIZE) ? -1.0 : 1.0;
    double c_norm_inf = 1.0;                                                /* :153-159 */
    for (int32_t j = 0; j < n; ++j) {
        c[j] = obj_sign * obj[j];
        c_norm_inf = maxd(c_norm_inf, fabs(c[j]));
    }
    double b_norm_inf = 1.0;                                                /* :160-167 */
    for (int32_t i = 0; i < m; ++i) {
        b_lo[i] = lo_sentinel(rlo[i]);
        b_hi[i] = hi_sentinel(rhi[i]);
        if (fabs(b_lo[i]) < 1e299) b_norm_inf = maxd(b_norm_inf, fabs(b_lo[i]));
        if (fabs(b_hi[i]) < 1e299) b_norm_inf = maxd(b_norm_inf, fabs(b_hi[i]));
    }
    for (int32_t col = 0; col < n; ++col)                                   /* :168-176 */
        for (int32_t p = lp->col_start[col]; p < lp->col_start[col + 1]; ++p) {
            const double v = fabs(val[p]);
            col_norms[col] += v;
            row_norms[lp->row_index[p]] += v;
        }
    for (int32_t j = 0; j < n; ++j) if (col_norms[j] < 1e-12) col_norms[j] = 1.0;
    for (int32_t i = 0; i < m; ++i) if (row_norms[i] < 1e-12) row_norms[i] = 1.0;
    double omega = (o->initial_primal_weight > 0.0)                         /* :177-178 */
                       ? o->initial_primal_weight
                       : clampd(sqrt(c_norm_inf / b_norm_inf), 0.01, 100.0);
    double eta = clampd(o->step_size_reduction, 0.1, 0.99);                 /* :179 */
#define UPDATE_STEP_SIZES()                                                   \
    do {                                                                      \
        for (int32_t j_ = 0; j_ < n; ++j_) tau[j_] = (eta / omega) / col_norms[j_]; \
        for (int32_t i_ = 0; i_ < m; ++i_) sigma[i_] = (eta * omega) / row_norms[i_]; \
    } while (0)
    UPDATE_STEP_SIZES();                                                    /* :180-185 */
    for (int32_t j = 0; j < n; ++j) {                                       /* :186-191 */
        double start = 0.0;
        if (initial_primal) start = initial_primal[j] * (ruiz ? 1.0 / col_scale[j] : 1.0);
        x[j] = clampd(start, lo_sentinel(vlo[j]), hi_sentinel(vhi[j]));
        x_bar[j] = x[j];
        x_avg[j] = x[j];
    }
    if (initial_dual)
        for (int32_t i = 0; i < m; ++i) {
            y[i] = initial_dual[i] * (ruiz ? 1.0 / row_scale[i] : 1.0);
            y_avg[i] = y[i];
        }
    int64_t iter = 0, avg_count = 0, iters_since_restart = 0;              /* :192-193 */
    double primal_infeas = 1e300, dual_infeas = 1e300, gap_val = 1e300, last_restart_score = 1e300;
    const int32_t* cs = lp->col_start;
    const int32_t* ri = lp->row_index;
    while (iter < o->max_iterations) {                                      /* :194 */
        oracle_spmv_t(m, n, cs, ri, val, y, At_y);                          /* :195 */
        memcpy(x_prev, x, sizeof(double) * (size_t)n);                     /* :196 */
        double dx_norm_sq = 0.0;
        for (int32_t j = 0; j < n; ++j) {                                   /* :198-205 */
            const double g = c[j] + At_y[j];
            const double proj_x = clampd(x[j] - tau[j] * g, lo_sentinel(vlo[j]), hi_sentinel(vhi[j]));
            const double dx = proj_x - x[j];
            delta_x[j] = dx;
            dx_norm_sq += col_norms[j] * dx * dx;
            x[j] = proj_x;
        }
        for (int32_t j = 0; j < n; ++j) x_bar[j] = 2.0 * x[j] - x_prev[j];  /* :206 */
        if (o->adaptive_step_size && iter % 10 == 0 && dx_norm_sq > 1e-14) { /* :207-219 */
            oracle_spmv(m, n, cs, ri, val, delta_x, Ax);
            double Adx_norm_sq = 0.0;
            for (int32_t i = 0; i < m; ++i) Adx_norm_sq += (Ax[i] * Ax[i]) / row_norms[i];
            if (Adx_norm_sq > 1e-14) {
                const double L_local = sqrt(Adx_norm_sq / dx_norm_sq);
                if (L_local > 1e-6) {
                    const double target_eta = 0.95 / L_local;
                    if (target_eta < eta) {
                        eta = maxd(0.1, maxd(target_eta, eta * 0.8));
                        UPDATE_STEP_SIZES();
                    } else if (target_eta > 1.05 * eta && eta < 0.99) {
                        eta = mind(0.99, eta * 1.05);
                        UPDATE_STEP_SIZES();
                    }
                }
            }
        }
        oracle_spmv(m, n, cs, ri, val, x_bar, Ax);                          /* :220 */
        for (int32_t i = 0; i < m; ++i) {                                   /* :221-224 */
            const double v = y[i] + sigma[i] * Ax[i];
            y[i] = v - sigma[i] * clampd(v / sigma[i], b_lo[i], b_hi[i]);
        }
        ++avg_count;                                                        /* :225-227 */
        for (int32_t j = 0; j < n; ++j) x_avg[j] += (x[j] - x_avg[j]) / (double)avg_count;
        for (int32_t i = 0; i < m; ++i) y_avg[i] += (y[i] - y_avg[i]) / (double)avg_count;
        ++iter;
        ++iters_since_restart;
        if (iter % o->restart_every == 0) {                                 /* :229-261 */
            oracle_spmv(m, n, cs, ri, val, x_avg, Ax);
            oracle_spmv_t(m, n, cs, ri, val, y_avg, At_y);
            const residuals_t cur = unscaled_residuals(lp, x_avg, y_avg, Ax, At_y, row_scale,
                                                       col_scale, ruiz, xu, yu);
            primal_infeas = cur.primal_infeas;
            dual_infeas = cur.dual_infeas;
            gap_val = cur.duality_gap;
            int restarted = 0;
            if (primal_infeas <= o->primal_tolerance && dual_infeas <= o->dual_tolerance &&
                gap_val <= o->gap_tolerance) {
                if (trace && trace->count < trace->capacity) {
                    const int64_t t = trace->count++;
                    trace->iteration[t] = iter;
                    trace->primal_infeasibility[t] = primal_infeas;
                    trace->dual_infeasibility[t] = dual_infeas;
                    trace->duality_gap[t] = gap_val;
                    trace->step_size[t] = eta;
                    trace->primal_weight[t] = omega;
                    trace->restarted[t] = 0;
                }
                const double elapsed = now_ms() - t_start;
                result->status = MC_PDLP_OPTIMAL;
                if (primal_out) memcpy(primal_out, xu, sizeof(double) * (size_t)n);
                if (dual_out) memcpy(dual_out, yu, sizeof(double) * (size_t)m);
                result->objective = cur.objective;
                result->primal_infeasibility = primal_infeas;
                result->dual_infeasibility = dual_infeas;
                result->duality_gap = gap_val;
                result->tolerance = o->primal_tolerance;
                result->iterations = iter;
                set_message(result, "PDLP converged");
                result->kernel_ms = elapsed;
                result->total_ms = elapsed;
                result->final_primal_weight = omega;
                result->final_step_size = eta;
                goto done;
            }
            const double current_score = cur.score;
            const int do_restart =
                (o->restart_strategy == MC_RESTART_FIXED) ||
                (o->restart_strategy == MC_RESTART_ADAPTIVE &&
                 (current_score <= o->restart_reduction_factor * last_restart_score ||
                  (iters_since_restart >= 5 * o->restart_every && current_score < last_restart_score)));
            if (do_restart) {
                if (o->adaptive_primal_weight && primal_infeas > 1e-12 && dual_infeas > 1e-12) {
                    const double ratio = clampd(sqrt(primal_infeas / dual_infeas), 0.05, 20.0);
                    omega = clampd(omega * pow(ratio, o->primal_weight_smoothing), 1e-6, 1e6);
                    UPDATE_STEP_SIZES();
                }
                memcpy(x, x_avg, sizeof(double) * (size_t)n);
                memcpy(y, y_avg, sizeof(double) * (size_t)m);
                memcpy(x_bar, x, sizeof(double) * (size_t)n);
                avg_count = 0;
                iters_since_restart = 0;
                last_restart_score = current_score;
                restarted = 1;
                result->restarts++;
            }
            if (trace && trace->count < trace->capacity) {
                const int64_t t = trace->count++;
                trace->iteration[t] = iter;
                trace->primal_infeasibility[t] = primal_infeas;
                trace->dual_infeasibility[t] = dual_infeas;
                trace->duality_gap[t] = gap_val;
                trace->step_size[t] = eta;
                trace->primal_weight[t] = omega;
                trace->restarted[t] = restarted;
            }
        }
    }
    {                                                                       /* :263-275 */
        oracle_spmv(m, n, cs, ri, val, x_avg, Ax);
        oracle_spmv_t(m, n, cs, ri, val, y_avg, At_y);
        const residuals_t fin = unscaled_residuals(lp, x_avg, y_avg, Ax, At_y, row_scale,
                                                   col_scale, ruiz, xu, yu);
        const double elapsed = now_ms() - t_start;
        result->status = MC_PDLP_ITERATION_LIMIT;
        if (primal_out) memcpy(primal_out, xu, sizeof(double) * (size_t)n);
        if (dual_out) memcpy(dual_out, yu, sizeof(double) * (size_t)m);
        result->objective = fin.objective;
        result->primal_infeasibility = fin.primal_infeas;
        result->dual_infeasibility = fin.dual_infeas;
        result->duality_gap = fin.duality_gap;
        result->tolerance = o->primal_tolerance;
        result->iterations = iter;
        set_message(result, "iteration limit reached");
        result->kernel_ms = elapsed;
        result->total_ms = elapsed;
        result->final_primal_weight = omega;
        result->final_step_size = eta;
    }
#undef UPDATE_STEP_SIZES
done:
    free(val); free(obj); free(vlo); free(vhi); free(rlo); free(rhi); free(row_scale);
    free(col_scale); free(c); free(b_lo); free(b_hi); free(row_norms); free(col_norms);
    free(tau); free(sigma); free(x); free(x_prev); free(x_bar); free(x_avg); free(delta_x);
    free(y); free(y_avg); free(At_y); free(Ax); free(xu); free(yu);
    return rc;
}
