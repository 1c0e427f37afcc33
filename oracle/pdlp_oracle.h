/*
 * CPU oracle for the PDLP engine -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's first-order LP path:
 *   equilibrate_model      src/scale/ruiz_scaling.cpp:152-247
 *   spmv / spmv_t          src/lp/first_order/pdlp.cpp:22-44
 *   compute_unscaled_residuals  src/lp/first_order/pdlp.cpp:62-135
 *   solve_pdlp             src/lp/first_order/pdlp.cpp:139-276
 * with the same operation order, so that built with the same compiler flags it
 * reproduces the reference bit for bit (pinned by tests against the reference
 * itself, compiled from its sources into oracle/_ref, and against the
 * committed golden vectors in tests/golden).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * call this code, and only as the checker.  The product never links it.
 */
#ifndef MC_PDLP_ORACLE_H
#define MC_PDLP_ORACLE_H

#include "mc_pdlp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Ruiz equilibration in place on a private copy; see the file header. */
int oracle_equilibrate(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                       double* value, double* objective, double* var_lower, double* var_upper,
                       double* row_lower, double* row_upper, int64_t max_iterations,
                       double tolerance, double* row_scale, double* col_scale,
                       int64_t* iterations_executed, int32_t* converged);

/* y = A x (CSC scatter, skips x_j == 0) and z = A^T y (column dots). */
void oracle_spmv(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                 const double* value, const double* x, double* y);
void oracle_spmv_t(int32_t m, int32_t n, const int32_t* col_start, const int32_t* row_index,
                   const double* value, const double* y, double* z);

/* Full solve.  Fills primal_out[n], dual_out[m] (may be NULL), result, and
 * the optional per-check trace. Returns MC_OK or MC_ERR_INVALID_ARGUMENT. */
int oracle_solve_pdlp(const mc_lp* lp, const mc_pdlp_options* options,
                      const double* initial_primal, const double* initial_dual,
                      double* primal_out, double* dual_out, mc_pdlp_result* result,
                      mc_pdlp_trace* trace);

#ifdef __cplusplus
}
#endif

#endif
