/*
 * mc_pdlp.h -- C ABI of the B200 (sm_100a) PDLP engine.
 *
 * This is the boundary a host solver binds to.  It replaces, for the GPU
 * backend, the reference entry
 *     PdlpResult solve_pdlp(const model::Model&, const PdlpOptions&)
 *     (include/markov_cero/lp/first_order/pdlp.hpp:67, src/lp/first_order/pdlp.cpp:139)
 * with plain pointers and sizes: no C++ types, no exceptions, an int status on
 * every call.  Options and results mirror PdlpOptions (pdlp.hpp:18-41) and
 * PdlpResult (pdlp.hpp:45-63) field by field; fields the reference does not
 * have are grouped at the end of each struct and say so.
 *
 * Model layout (model.hpp:25-34, 53-70): CSC with int32 column pointers and
 * row indices (rows strictly increasing within a column, values finite and
 * nonzero, exactly what SparseMatrixCSC::validate accepts, model.cpp:41-66)
 * and +-INFINITY in place of BoundKind::{negative,positive}_infinity.
 *
 * Threading: calls on different contexts may run concurrently from different
 * host threads; one context must not be used by two threads at once.
 * Errors: every function returns MC_OK (0) or an mc_error code; the text of
 * the last error on the calling thread is available from mc_last_error().
 * There is no CPU fallback: without a usable sm_100 device every solve
 * returns MC_ERR_NO_DEVICE.
 */
#ifndef MC_PDLP_H
#define MC_PDLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC_PDLP_ABI_VERSION 1

/* Return codes of every entry point. The CLI of the reference maps
 * std::invalid_argument -> InvalidModel, std::length_error -> ResourceLimit and
 * anything else -> NumericalFailure (apps/markov_cero_solve.cpp:418-434); the
 * codes below keep those three classes apart. */
typedef enum mc_error {
    MC_OK = 0,
    MC_ERR_INVALID_ARGUMENT = 1, /* malformed model/options (invalid_argument) */
    MC_ERR_NO_DEVICE = 2,        /* no CUDA device, or not sm_100             */
    MC_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed                  */
    MC_ERR_RESOURCE_LIMIT = 4,   /* sizes beyond the engine's index range     */
    MC_ERR_CUDA = 5,             /* any other CUDA runtime error              */
    MC_ERR_INTERNAL = 6
} mc_error;

/* PdlpStatus, same order (pdlp.hpp:43). */
typedef enum mc_pdlp_status {
    MC_PDLP_OPTIMAL = 0,
    MC_PDLP_ITERATION_LIMIT = 1,
    MC_PDLP_INFEASIBLE_OR_UNBOUNDED = 2,
    MC_PDLP_NUMERICAL_FAILURE = 3
} mc_pdlp_status;

enum { MC_BACKEND_CPU = 0, MC_BACKEND_GPU = 1 };                 /* pdlp.hpp:15 */
enum { MC_RESTART_NONE = 0, MC_RESTART_ADAPTIVE = 1, MC_RESTART_FIXED = 2 }; /* pdlp.hpp:16 */
enum { MC_MINIMIZE = 0, MC_MAXIMIZE = 1 };                       /* model.hpp:11 */
enum { MC_MEMORY_HOST = 0, MC_MEMORY_DEVICE = 1 };
enum { MC_PRECISION_FP64 = 0, MC_PRECISION_FP32_REFINE = 1 };

/* An LP in the reference's Model shape (model.hpp:53-70).  `memory` says
 * where every array lives; device arrays must belong to the context's
 * device.  The engine never writes to these arrays. */
typedef struct mc_lp {
    int32_t num_rows;            /* m */
    int32_t num_cols;            /* n */
    int64_t nnz;
    const int32_t* col_start;    /* [n+1], col_start[0] = 0, col_start[n] = nnz */
    const int32_t* row_index;    /* [nnz] */
    const double* value;         /* [nnz] */
    const double* objective;     /* [n] */
    const double* var_lower;     /* [n], -INFINITY = unbounded below */
    const double* var_upper;     /* [n], +INFINITY = unbounded above */
    const double* row_lower;     /* [m] */
    const double* row_upper;     /* [m] */
    double objective_offset;
    int32_t objective_sense;     /* MC_MINIMIZE / MC_MAXIMIZE */
    int32_t memory;              /* MC_MEMORY_HOST / MC_MEMORY_DEVICE */
} mc_lp;

/* PdlpOptions (pdlp.hpp:18-41). Defaults from mc_pdlp_default_options(). */
typedef struct mc_pdlp_options {
    int64_t max_iterations;           /* 100000 */
    int64_t restart_every;            /* 40 */
    double primal_tolerance;          /* 1e-4 */
    double dual_tolerance;            /* 1e-4 */
    double gap_tolerance;             /* 1e-4 */
    double step_size_reduction;       /* 0.9 (initial eta) */
    int64_t power_iterations;         /* 20, unused (as in the reference) */
    int32_t backend;                  /* MC_BACKEND_GPU; MC_BACKEND_CPU is rejected */
    int32_t restart_strategy;         /* MC_RESTART_ADAPTIVE */
    double restart_reduction_factor;  /* 0.368 */
    int32_t adaptive_step_size;       /* 1 */
    int32_t adaptive_primal_weight;   /* 1 */
    double initial_primal_weight;     /* 0 = derive from ||c|| / ||b|| */
    double primal_weight_smoothing;   /* 0.5 */
    int32_t ruiz_scaling;             /* 1 */
    int64_t ruiz_iterations;          /* 10 */
    /* ---- engine extensions, no counterpart in PdlpOptions ---- */
    int32_t precision;                /* MC_PRECISION_FP64 */
    int32_t device;                   /* CUDA ordinal used by mc_pdlp_solve, default 0 */
    int32_t profile_kernels;          /* 1: time every kernel launch with CUDA events
                                         (no CUDA graph; slower); fills kernel_ms_by_kind */
    int32_t check_every_chunks;       /* host status poll interval in restart chunks, default 1 */
    int32_t lanes_per_column;         /* A^T y kernel: 0 = automatic (single LP: by mean
                                         column length; batch: the lanes autotuner, timed on
                                         the batch and kept per context and batch shape),
                                         1..32 (power of two) = lanes per column */
    int32_t lanes_per_row;            /* A x kernel, same meaning per row */
    int32_t warm_start_guard;         /* 1: with a warm start, evaluate the reference's KKT score
                                         of the warm start and of the cold start (x = proj(0),
                                         y = 0) on the device and run from the better one; a
                                         cold start also drops initial_primal_weight */
    int32_t reserved_i[4];
    double reserved_d[8];
} mc_pdlp_options;

enum {
    MC_KERNEL_PRIMAL = 0,    /* A^T y SpMV + primal prox + averages           */
    MC_KERNEL_DUAL = 1,      /* A x-bar SpMV + dual prox + averages           */
    MC_KERNEL_DUAL_STEP = 2, /* A x-bar and A dx SpMV on step-size iterations */
    MC_KERNEL_RESIDUAL = 3,  /* KKT residual SpMVs + reductions + restart     */
    MC_KERNEL_SETUP = 4,     /* transpose, Ruiz, norms                        */
    MC_KERNEL_OTHER = 5,
    MC_KERNEL_KINDS = 8
};

/* PdlpResult (pdlp.hpp:45-63).  primal/dual are returned through separate
 * caller-owned buffers (see mc_pdlp_solve). */
typedef struct mc_pdlp_result {
    int32_t status;                   /* mc_pdlp_status */
    double objective;
    double primal_infeasibility;
    double dual_infeasibility;
    double duality_gap;
    double tolerance;
    int64_t iterations;
    char message[160];
    double h2d_ms;
    double kernel_ms;
    double d2h_ms;
    double total_ms;
    char backend_actually_used[16];   /* "cuda" */
    /* ---- engine extensions ---- */
    int64_t ruiz_iterations_executed;
    int64_t restarts;
    double final_primal_weight;
    double final_step_size;           /* eta */
    int64_t refinement_rounds;        /* FP32_REFINE only */
    int64_t inner_iterations;         /* FP32_REFINE: PDHG iterations over all rounds */
    double kernel_ms_by_kind[MC_KERNEL_KINDS];
    int64_t launches_by_kind[MC_KERNEL_KINDS];
    int64_t kernel_launches;          /* engine kernels launched by this solve */
    int32_t warm_start_used;          /* 1 if the solve started from the given warm start */
    int32_t certificate;              /* batched solves, status INFEASIBLE_OR_UNBOUNDED: the
                                         mc_certificate kind that proves it (else MC_CERT_NONE) */
    double warm_start_score;          /* guard: max(primal, dual, gap) at the warm start */
    double cold_start_score;          /* guard: the same at the cold start */
    int64_t certificate_index;        /* MC_CERT_CROSSED_BOUNDS: the column; MC_CERT_ROW_ACTIVITY:
                                         the row (indices of the LP itself); else -1 */
    double reserved_d1;
} mc_pdlp_result;

/* Infeasibility certificates of batched solves (no counterpart in the
 * reference, whose PDLP never returns INFEASIBLE_OR_UNBOUNDED, pdlp.hpp:43).
 * Each proves that no x satisfies row_lower <= A x <= row_upper and
 * var_lower <= x <= var_upper:
 *   CROSSED_BOUNDS: var_lower[j] > var_upper[j] for j = certificate_index.
 *   ROW_ACTIVITY:   row i = certificate_index cannot be met with every variable
 *                   in its box: max over the box of (A x)_i < row_lower[i], or
 *                   min > row_upper[i] (a dual ray y = -e_i or +e_i).
 *   DUAL_RAY:       dual_out holds a ray y (unscaled, the reference's sign
 *                   convention: y_i > 0 only on rows with a finite upper
 *                   bound, y_i < 0 only with a finite lower bound) with
 *                   g = A^T y and
 *                     L = sum_j (g_j > 0 ? g_j var_lower[j] : g_j var_upper[j])
 *                     U = sum_i (y_i > 0 ? y_i row_upper[i] : y_i row_lower[i])
 *                   all finite and L > U; for every x in the box
 *                   L <= g.x = y.(A x) <= U would hold if x were feasible.
 *                   Found by the restart checks: the change of the dual
 *                   average between two checks, with its components on
 *                   one-sided rows projected to the allowed sign -- the dual
 *                   iterates of a primal infeasible LP diverge along a ray. */
enum {
    MC_CERT_NONE = 0,
    MC_CERT_CROSSED_BOUNDS = 1,
    MC_CERT_ROW_ACTIVITY = 2,
    MC_CERT_DUAL_RAY = 3
};

/* Optional per-check history (one entry per restart check). */
typedef struct mc_pdlp_trace {
    int64_t capacity;   /* entries available in every array below */
    int64_t count;      /* entries written */
    int64_t* iteration;
    double* primal_infeasibility;
    double* dual_infeasibility;
    double* duality_gap;
    double* step_size;       /* eta after the check */
    double* primal_weight;   /* omega after the check */
    int32_t* restarted;
} mc_pdlp_trace;

typedef struct mc_pdlp_ctx mc_pdlp_ctx;

int mc_pdlp_abi_version(void);
void mc_pdlp_default_options(mc_pdlp_options* options);

/* sizeof of mc_lp, mc_pdlp_options, mc_pdlp_result, mc_pdlp_trace,
 * mc_verify_report, mc_canonical_lp, mc_presolve_options, mc_presolve_info
 * (in that order) into sizes[0..count-1]; lets bindings check their struct
 * layouts. */
int mc_pdlp_struct_sizes(size_t* sizes, int count);

/* Thread-local text of the last failure ("" if none). Returns MC_OK. */
int mc_last_error(char* buffer, size_t length);

/* Number of usable sm_100 devices (0 if none). */
int mc_device_count(int* count);

/* A context owns a device, a stream and reusable device buffers; keeping one
 * alive across solves avoids repeated allocation. */
int mc_pdlp_ctx_create(int device, mc_pdlp_ctx** out);
int mc_pdlp_ctx_destroy(mc_pdlp_ctx* ctx);

/*
 * Solve one LP with PDLP on the GPU.  Same algorithm, options, statuses and
 * result fields as the reference solve_pdlp (src/lp/first_order/pdlp.cpp:139-276):
 * Ruiz equilibration, diagonal steps, adaptive step size, adaptive restarts
 * to the average, adaptive primal weight, relative KKT termination on the
 * unscaled averages, checked every restart_every iterations.
 *   initial_primal / initial_dual: optional warm start in the original space
 *     (NULL = the reference start x = proj(0), y = 0); an extension.
 *   primal_out[n] / dual_out[m]: caller-owned, in lp->memory space; receive the
 *     unscaled average iterates, like PdlpResult::primal / dual.  May be NULL.
 *   trace: optional history, may be NULL.
 * Non-convergence is a status, not an error.
 */
int mc_pdlp_ctx_solve(mc_pdlp_ctx* ctx, const mc_lp* lp, const mc_pdlp_options* options,
                      const double* initial_primal, const double* initial_dual,
                      double* primal_out, double* dual_out,
                      mc_pdlp_result* result, mc_pdlp_trace* trace);

/* The context's CUDA stream (a cudaStream_t), on which every kernel of the
 * context runs: callers time the engine with CUDA events recorded on it. */
int mc_pdlp_ctx_stream(mc_pdlp_ctx* ctx, void** stream);

/*
 * Stepwise form of mc_pdlp_ctx_solve: the same solve driven a few restart
 * chunks at a time, so that a caller can time, interleave or stop the PDHG
 * loop (pdlp.cpp:194-262) between chunks.  The reference's solve_pdlp runs
 * the loop in one call; begin + iterate (to the end) + finish gives the same
 * result as mc_pdlp_ctx_solve, bit for bit.
 *   mc_pdlp_ctx_begin:   everything before the first iteration (uploads,
 *                        validation, transpose, Ruiz, norms, start point,
 *                        pdlp.cpp:139-191); arguments as mc_pdlp_ctx_solve.
 *                        Host arrays of `lp` are copied during the call; device
 *                        arrays (and `trace`) must stay valid until finish.
 *   mc_pdlp_ctx_iterate: up to `chunks` further chunks (each restart_every
 *                        iterations and the restart check); returns with the
 *                        context's stream synchronised.  *iterations (may be
 *                        NULL): iterations done so far; *finished (may be
 *                        NULL): 1 once the solve has converged, failed or
 *                        reached max_iterations' last whole chunk.
 *   mc_pdlp_ctx_finish:  the remaining partial chunk and final evaluation if
 *                        the loop reached max_iterations (pdlp.cpp:263-265),
 *                        then outputs and result as mc_pdlp_ctx_solve.  A solve
 *                        finished early reports iteration_limit with the last
 *                        check's averages, as a solve with max_iterations set
 *                        to the iterations done would.
 * One solve in progress per context: any other solve, batch or verify call on
 * the context ends it (iterate / finish then return MC_ERR_INVALID_ARGUMENT).
 */
int mc_pdlp_ctx_begin(mc_pdlp_ctx* ctx, const mc_lp* lp, const mc_pdlp_options* options,
                      const double* initial_primal, const double* initial_dual,
                      mc_pdlp_trace* trace);
int mc_pdlp_ctx_iterate(mc_pdlp_ctx* ctx, int64_t chunks, int64_t* iterations, int32_t* finished);
int mc_pdlp_ctx_finish(mc_pdlp_ctx* ctx, double* primal_out, double* dual_out,
                       mc_pdlp_result* result);

/* One-shot form: a temporary context on options->device. */
int mc_pdlp_solve(const mc_lp* lp, const mc_pdlp_options* options,
                  const double* initial_primal, const double* initial_dual,
                  double* primal_out, double* dual_out, mc_pdlp_result* result);

/*
 * Batched solve: `count` independent LPs of any sizes in one set of launches
 * (no counterpart in the reference, which solves one LP per call).  The LPs
 * are packed block-diagonally on the device and every LP runs the same
 * algorithm as mc_pdlp_ctx_solve with its own step size, primal weight,
 * restarts and termination.  Each lps[b] may be in host or device memory
 * (its `memory` field); primal_out[b] / dual_out[b] (arrays of `count`
 * pointers, entries may be NULL) receive the unscaled averages of LP b in
 * the same memory space as lps[b].  results[b] is LP b's result.  An LP with
 * a crossed bound (lower > upper) or a row whose activity interval over the
 * variable box misses the row's bounds is reported
 * MC_PDLP_INFEASIBLE_OR_UNBOUNDED at setup.  FP64 form only.
 */
int mc_pdlp_ctx_solve_batch(mc_pdlp_ctx* ctx, const mc_lp* lps, int32_t count,
                            const mc_pdlp_options* options, double* const* primal_out,
                            double* const* dual_out, mc_pdlp_result* results);

/* The batched solve with a starting point per LP, as initial_primal /
 * initial_dual of mc_pdlp_ctx_solve (original space; projected onto the
 * bounds): initial_primal[b] (num_cols of LP b) and initial_dual[b] (num_rows),
 * either array or any entry NULL for a cold start of that part.  Branch and
 * bound passes each node the parent's solution.  No guard: the start is used
 * as given (warm_start_guard is ignored).  No counterpart in the reference,
 * whose node LPs warm-start the dual simplex from the parent's basis
 * (src/milp/node_lp.cpp:44-60). */
int mc_pdlp_ctx_solve_batch_warm(mc_pdlp_ctx* ctx, const mc_lp* lps, int32_t count,
                                 const mc_pdlp_options* options, const double* const* initial_primal,
                                 const double* const* initial_dual, double* const* primal_out,
                                 double* const* dual_out, mc_pdlp_result* results);

/*
 * Variants of one LP that differ only in their variable bounds -- the nodes
 * of one branching round of branch and bound, which tighten bounds of the
 * parent LP (src/milp/milp_solver.cpp:401-447) -- solved together with the
 * matrix read once per iteration for all of them (no counterpart in the
 * reference, which solves one node LP per call, src/milp/node_lp.cpp:9-82).
 * `base` gives A, the objective, the row bounds and default variable bounds;
 * variant b replaces the variable bounds by var_lower[b] / var_upper[b]
 * (num_cols each, host or device memory; a NULL array or entry keeps the
 * base's).  initial_primal / initial_dual (may be NULL, or hold NULL
 * entries) give starting points in original units, as for
 * mc_pdlp_ctx_solve_batch_warm.  Every variant runs the algorithm of
 * mc_pdlp_ctx_solve on its own LP (own step size, primal weight, restarts,
 * termination); results[b], primal_out[b] / dual_out[b] (may be NULL) as for
 * the batch.  Infeasible variants end with INFEASIBLE_OR_UNBOUNDED and a
 * certificate (crossed bounds, row activity, or a dual ray in dual_out[b]).
 * Both precision forms: MC_PRECISION_FP32_REFINE runs each variant as an
 * FP64 base plus an FP32 correction, re-centred at every restart, as the
 * single-LP form does.
 */
int mc_pdlp_ctx_solve_variants(mc_pdlp_ctx* ctx, const mc_lp* base, int32_t count,
                               const double* const* var_lower, const double* const* var_upper,
                               const mc_pdlp_options* options, const double* const* initial_primal,
                               const double* const* initial_dual, double* const* primal_out,
                               double* const* dual_out, mc_pdlp_result* results);

/*
 * Learned warm start (no counterpart in the reference): a bipartite
 * message-passing network over an LP's constraint/variable graph (hidden 64,
 * `rounds` rounds, FP32) that predicts a primal/dual starting point and the
 * log of the initial primal weight.  Trained and run on the GPU by the
 * engine's own forward/backward kernels.  LPs are read from host memory.
 * Feed the prediction to mc_pdlp_ctx_solve as initial_primal / initial_dual
 * with warm_start_guard = 1, which falls back to the cold start whenever the
 * prediction's KKT score is worse.  Leave initial_primal_weight at 0 (the
 * derived weight): the predicted weight cost iterations in measurement.
 */
typedef struct mc_gnn mc_gnn;
int mc_gnn_create(int device, int rounds, uint64_t seed, mc_gnn** out);
int mc_gnn_destroy(mc_gnn* net);
int mc_gnn_num_params(const mc_gnn* net, int64_t* count);
int mc_gnn_get_params(mc_gnn* net, float* params_out);
int mc_gnn_set_params(mc_gnn* net, const float* params_in);
/* x_out[n], y_out[m] in the LP's original units; *log_omega_out (may be NULL) */
int mc_gnn_predict(mc_gnn* net, const mc_lp* lp, double* x_out, double* y_out, double* log_omega_out);
/* loss against a solved instance (x*, y*, log omega*) and its gradient
 * (grad_out[num_params], may be NULL) */
int mc_gnn_loss_and_grad(mc_gnn* net, const mc_lp* lp, const double* x_target, const double* y_target,
                         double log_omega_target, double* loss, float* grad_out);
/* one Adam step (beta 0.9 / 0.999) on one instance; *loss before the step */
int mc_gnn_train_step(mc_gnn* net, const mc_lp* lp, const double* x_target, const double* y_target,
                      double log_omega_target, float learning_rate, double* loss);

/*
 * Kernel-level entry points (device pointers, the context's stream), used by
 * the parity tests and the roofline measurement.  They replace the reference's
 * file-local helpers of the same meaning.
 */

/* y = A x over CSR (row_start[m+1], col_index, value); the reference computes
 * it as a CSC scatter, spmv() at src/lp/first_order/pdlp.cpp:22-32. */
int mc_spmv_csr(mc_pdlp_ctx* ctx, int32_t m, int32_t n, const int32_t* row_start,
                const int32_t* col_index, const double* value, const double* x, double* y);

/* Build CSR(A) from CSC(A) on the device, rows' entries in ascending column
 * order; the reference keeps only CSC.  row_start[m+1], col_index[nnz],
 * value[nnz] are caller-allocated device arrays. */
int mc_csc_to_csr(mc_pdlp_ctx* ctx, int32_t m, int32_t n, int64_t nnz,
                  const int32_t* col_start, const int32_t* row_index, const double* value,
                  int32_t* row_start, int32_t* col_index, double* csr_value);

/* Ruiz equilibration of a device-resident model in place (values of both
 * copies, bounds, objective), equilibrate_model at
 * src/scale/ruiz_scaling.cpp:152-247.  row_scale[m], col_scale[n] receive D_R,
 * D_C; *iterations_executed the pass count. */
int mc_ruiz_equilibrate(mc_pdlp_ctx* ctx, int32_t m, int32_t n, int64_t nnz,
                        const int32_t* col_start, const int32_t* row_index, double* csc_value,
                        const int32_t* row_start, const int32_t* col_index, double* csr_value,
                        double* objective, double* var_lower, double* var_upper,
                        double* row_lower, double* row_upper, int64_t max_iterations,
                        double* row_scale, double* col_scale, int64_t* iterations_executed);

/* The simplex path's equilibration of a canonical model (SparseCanonicalModel
 * CSC, rhs, objective) on the device: equilibrate at
 * src/scale/ruiz_scaling.cpp:20-125.  The same Ruiz loop as above with the
 * given tolerance, then the scales clamped to [min_scale, max_scale] (values
 * keep the unclamped scaling, as in the reference), their inverses, rhs[m]
 * scaled by the row scales and objective[n] by the column scales.  An empty
 * model (m, n or nnz 0) gets unit scales and untouched rhs/objective.  A
 * non-finite scaled rhs/objective is MC_ERR_INVALID_ARGUMENT (the reference
 * throws overflow_error).  Device arrays; reference defaults: 10 passes,
 * tolerance 1e-3, scales in [1e-4, 1e4]. */
int mc_ruiz_equilibrate_canonical(mc_pdlp_ctx* ctx, int32_t m, int32_t n, int64_t nnz,
                                  const int32_t* col_start, const int32_t* row_index, double* value,
                                  double* rhs, double* objective, int64_t max_iterations, double tolerance,
                                  double min_scale, double max_scale, double* row_scale, double* col_scale,
                                  double* inv_row_scale, double* inv_col_scale, int64_t* iterations_executed,
                                  int32_t* converged);

/*
 * Post-solve verification of a primal candidate on the device, verify_primal
 * at src/verify/primal_verifier.cpp:44-103 as the CLI calls it after a PDLP
 * solve (apps/markov_cero_solve.cpp:164-168): variable bounds, row activities
 * A x against the row bounds, and the objective recomputed and compared with
 * the claimed one, each with an allowance abs + rel * max(1, |actual|,
 * |expected|).  Row activities are summed in the reference's order (ascending
 * column within each row) and, like the objective, in double-double
 * arithmetic where the reference uses long double.  Continuous models only
 * (mc_lp carries no integrality).
 */
typedef enum mc_violation_kind {
    MC_VIOLATION_VARIABLE_LOWER = 0,
    MC_VIOLATION_VARIABLE_UPPER = 1,
    MC_VIOLATION_ROW_LOWER = 2,
    MC_VIOLATION_ROW_UPPER = 3,
    MC_VIOLATION_OBJECTIVE = 4,
    MC_VIOLATION_KINDS = 5
} mc_violation_kind;

typedef struct mc_verify_report {
    int32_t passed;                    /* no violation of any kind */
    int32_t reserved0;
    double recomputed_objective;       /* offset + sum c_j x_j (original objective) */
    double objective_difference;       /* |recomputed - claimed| */
    double maximum_row_violation;
    double maximum_variable_violation;
    int64_t violations[MC_VIOLATION_KINDS];   /* count per kind */
    int64_t first_index[MC_VIOLATION_KINDS];  /* lowest violating index per kind, -1 if none */
    double reserved_d[4];
} mc_verify_report;

/* primal[num_cols] in the memory the lp's `memory` field names.  Tolerances as
 * the reference's Tolerance (finite, 0 <= value <= 1e-4, else
 * MC_ERR_INVALID_ARGUMENT); a non-finite candidate entry or claimed objective
 * is MC_ERR_INVALID_ARGUMENT, as the reference throws invalid_argument. */
int mc_verify_primal(mc_pdlp_ctx* ctx, const mc_lp* lp, const double* primal, double claimed_objective,
                     double feasibility_absolute, double feasibility_relative, double objective_absolute,
                     double objective_relative, mc_verify_report* report);

/*
 * Binary CSC model files ("MCLPCSC1": a 64-byte header, then col_start,
 * row_index, value, objective, var_lower, var_upper, row_lower, row_upper as
 * raw little-endian int32/double arrays; infinite bounds as IEEE infinities).
 * They carry models past the reference MPS reader's limits
 * (include/markov_cero/io/mps.hpp:13-20: 16 MiB, 1M rows or columns, 20M
 * nonzeros), which the config-1 to config-3 models exceed.  No counterpart in
 * the reference.
 *   mc_lp_file_write: lp->memory must be MC_MEMORY_HOST.
 *   mc_lp_file_info:  sizes from the header (the file length is checked).
 *   mc_lp_file_read:  fills the caller's arrays, sized by lp->num_rows /
 *     num_cols / nnz (must equal the file's), host or device per lp->memory
 *     (device arrays on the current device: streamed through two 8 MiB pinned
 *     buffers); sets objective_offset and objective_sense.  The arrays are
 *     validated by the solve that uses them.
 */
int mc_lp_file_write(const char* path, const mc_lp* lp);
int mc_lp_file_info(const char* path, int32_t* num_rows, int32_t* num_cols, int64_t* nnz);
int mc_lp_file_read(const char* path, mc_lp* lp);

/*
 * mc_ruiz_equilibrate_noalloc: the same equilibration as mc_ruiz_equilibrate,
 * with bit-identical results, for callers that cannot allocate device memory
 * (device memory all owned by another allocator such as a caching pool or a
 * fixed arena; a request path that must not allocate, since an allocation can
 * wait on the device for an unbounded time).  No counterpart in the reference.
 * It allocates nothing: its working memory is one static device array of
 * about 8 MiB that every GPU loading the library holds until exit.
 * Limits: m + n <= 1,048,576, else MC_ERR_RESOURCE_LIMIT (nothing launched).
 * Runs on the current device and `stream` (a cudaStream_t, NULL = default
 * stream).  With iterations_executed non-NULL the call reads the pass count
 * back with a stream synchronisation and reports errors of its kernels; with
 * it NULL the call returns once its work is enqueued, asynchronously on
 * `stream`, and errors that arise while the kernels run surface only in the
 * caller's own later checks of that stream.  The first call on a device looks
 * the array up with cudaGetSymbolAddress and keeps the address for the life
 * of the process: make that call before any stream capture, and do not call
 * on a device after cudaDeviceReset (the kept address belongs to the old
 * context).  Calls share the array, so calls that can overlap on the GPU race
 * and must be serialised.
 */
int mc_ruiz_equilibrate_noalloc(int32_t m, int32_t n, int64_t nnz, const int32_t* col_start,
                                const int32_t* row_index, double* csc_value,
                                const int32_t* row_start, const int32_t* col_index,
                                double* csr_value, double* objective, double* var_lower,
                                double* var_upper, double* row_lower, double* row_upper,
                                int64_t max_iterations, double* row_scale, double* col_scale,
                                int64_t* iterations_executed, void* stream);

/*
 * Presolve of a canonical model on the device: presolve() and postsolve() at
 * src/presolve/presolve.cpp:20-217 and :219-317 (options and statistics:
 * include/markov_cero/presolve/presolve.hpp:12-36; the record stack:
 * include/markov_cero/presolve/presolve_stack.hpp:9-72).
 *
 * The canonical model is SparseCanonicalModel (min c.x + offset, A x = rhs,
 * x >= 0; include/markov_cero/transform/sparse_canonical_model.hpp:12-19):
 * CSC with strictly increasing row indices in each column, no explicit zeros,
 * finite values, rhs and objective.  A model that breaks these is
 * MC_ERR_INVALID_ARGUMENT (the reference's validate() throws).  The
 * reference's dense-simplex size cap (4096 rows and columns, 4Mi nonzeros,
 * src/linalg/sparse_basis.cpp:26-34) is not applied: the device presolve
 * takes any model within the int32 index range.
 *
 * Each pass removes empty rows (row order), then empty columns (column
 * order), then row singletons in row order, each fixing its variable and
 * substituting it into the other rows -- with exactly the reference's
 * sequential semantics: a row left with one entry by an earlier singleton of
 * the same pass is itself a singleton, and right-hand sides are updated in
 * the reference's order, so the reduced model, the record stack and the maps
 * are bit-identical to the reference's.  Up to max_passes passes; stops after
 * a pass without reductions.
 *
 * Arrays of mc_canonical_lp may be host or device memory (cudaMemcpyDefault).
 */
typedef struct mc_canonical_lp {
    int32_t num_rows, num_cols;
    int64_t nnz;
    const int32_t* col_start; /* [num_cols + 1] */
    const int32_t* row_index; /* [nnz] */
    const double* value;      /* [nnz] */
    const double* rhs;        /* [num_rows] */
    const double* objective;  /* [num_cols] */
    double objective_offset;
} mc_canonical_lp;

typedef struct mc_presolve_options { /* PresolveOptions, presolve.hpp:12-17 */
    int64_t max_passes;              /* 5 */
    double feasibility_tolerance;    /* 1e-9 */
    double dual_tolerance;           /* 1e-9 */
    double pivot_tolerance;          /* 1e-12 */
} mc_presolve_options;

void mc_presolve_default_options(mc_presolve_options* options);

/* lp::reference::SolveStatus values that presolve returns */
typedef enum mc_presolve_status {
    MC_PRESOLVE_OPTIMAL = 0,    /* reduced ("presolve complete") */
    MC_PRESOLVE_INFEASIBLE = 1, /* an empty row with a non-zero rhs, or a negative singleton value */
    MC_PRESOLVE_UNBOUNDED = 2   /* an empty column with a negative cost */
} mc_presolve_status;

/* ReductionRecord alternatives, in the variant's order (presolve_stack.hpp:38-39) */
typedef enum mc_record_kind {
    MC_RECORD_EMPTY_ROW = 0,      /* index = row, value = rhs_value */
    MC_RECORD_EMPTY_COLUMN = 1,   /* index = column, value = objective_coeff, value2 = fixed_value */
    MC_RECORD_FIXED_VARIABLE = 2, /* index = column, value = fixed_value, value2 = objective_coeff;
                                     incident rows and coefficients */
    MC_RECORD_ROW_SINGLETON = 3   /* index = row, variable = column, value = coefficient, value2 = rhs_value */
} mc_record_kind;

typedef struct mc_presolve_info {
    int32_t status; /* mc_presolve_status */
    char message[96];
    /* PresolveStatistics, presolve.hpp:19-29 */
    int64_t passes_executed, empty_rows_removed, empty_cols_removed, fixed_vars_removed, row_singletons_removed;
    int64_t original_rows, original_cols, presolved_rows, presolved_cols;
    int64_t presolved_nnz;
    double objective_offset; /* of the reduced model */
    int64_t records;          /* stack size */
    int64_t incident_entries; /* rows over all fixed-variable records */
    int64_t scan_rounds;      /* device rounds of the singleton scans, over all passes */
    double presolve_ms;       /* host wall time of mc_presolve_run */
} mc_presolve_info;

typedef struct mc_presolve mc_presolve; /* a presolve's result, held in device memory */

/* Runs presolve on the context's device; *out receives the result (status
 * infeasible/unbounded are results, not errors).  Free with mc_presolve_free. */
int mc_presolve_run(mc_pdlp_ctx* ctx, const mc_canonical_lp* lp, const mc_presolve_options* options,
                    mc_presolve** out);
int mc_presolve_get_info(const mc_presolve* p, mc_presolve_info* info);
/* The reduced model (presolved_rows x presolved_cols, presolved_nnz): host or
 * device destinations; any pointer may be NULL.  Empty when status is not
 * optimal (the reference returns a default model then). */
int mc_presolve_get_model(const mc_presolve* p, int32_t* col_start, int32_t* row_index, double* value,
                          double* rhs, double* objective);
/* presolved_to_original rows [presolved_rows] and columns [presolved_cols] */
int mc_presolve_get_maps(const mc_presolve* p, int64_t* row_map, int64_t* col_map);
/* The stack, oldest first: kind, index, variable (-1 if none), value, value2
 * [records]; incident_start [records + 1] into incident_row and
 * incident_coefficient [incident_entries].  Any pointer may be NULL. */
int mc_presolve_get_records(const mc_presolve* p, int32_t* kind, int64_t* index, int64_t* variable, double* value,
                            double* value2, int64_t* incident_start, int64_t* incident_row,
                            double* incident_coefficient);
/* postsolve() against the model presolve ran on: reduced_primal
 * [reduced_cols] and reduced_dual [reduced_rows] (entries past a shorter
 * array count as missing, as in the reference); writes primal [num_cols],
 * dual [num_rows] and the objective.  The singleton duals and the objective
 * are summed in double-double arithmetic where the reference uses long
 * double.  A non-finite dual or objective is MC_ERR_INVALID_ARGUMENT (the
 * reference throws overflow_error). */
int mc_postsolve(mc_pdlp_ctx* ctx, const mc_presolve* p, const double* reduced_primal, int64_t reduced_cols,
                 const double* reduced_dual, int64_t reduced_rows, double* primal, double* dual, double* objective);
void mc_presolve_free(mc_presolve* p);
/* A presolve result rebuilt from a stack held by the caller (for a caller
 * that keeps the reference's PresolveStack, presolve_stack.hpp:41-72, and
 * wants mc_postsolve on it): `original` is the model presolve ran on, the
 * record arrays are as mc_presolve_get_records gives them (incident lists are
 * not needed by postsolve), the maps as mc_presolve_get_maps.  Host arrays.
 * Indices out of range or unknown kinds are MC_ERR_INVALID_ARGUMENT. */
int mc_presolve_load(mc_pdlp_ctx* ctx, const mc_canonical_lp* original, int64_t records, const int32_t* kind,
                     const int64_t* index, const int64_t* variable, const double* value, const double* value2,
                     int64_t presolved_rows, const int64_t* row_map, int64_t presolved_cols, const int64_t* col_map,
                     mc_presolve** out);

#ifdef __cplusplus
}
#endif

#endif /* MC_PDLP_H */
