/*
 * CPU oracle for the device presolve -- TEST INFRASTRUCTURE ONLY (see
 * presolve_oracle.c).  Restates src/presolve/presolve.cpp:20-317.
 */
#ifndef MC_PRESOLVE_ORACLE_H
#define MC_PRESOLVE_ORACLE_H

#include "mc_pdlp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Caller-allocated outputs at their largest sizes: the reduced model
 * (col_start [n+1], row_index / values [nnz], rhs [m], objective [n]), the
 * maps (row_map [m], col_map [n]) and the stack (kind ... value2 [m+n],
 * incident_start [m+n+1], incident_row / incident_coefficient [nnz]). */
typedef struct oracle_presolve_out {
    int32_t* col_start;
    int32_t* row_index;
    double* values;
    double* rhs;
    double* objective;
    int64_t* row_map;
    int64_t* col_map;
    int32_t* kind;
    int64_t* index;
    int64_t* variable;
    double* value;
    double* value2;
    int64_t* incident_start;
    int64_t* incident_row;
    double* incident_coefficient;
} oracle_presolve_out;

int oracle_presolve(const mc_canonical_lp* lp, const mc_presolve_options* options, mc_presolve_info* info,
                    oracle_presolve_out* out);

int oracle_postsolve(const mc_canonical_lp* lp, int64_t records, const int32_t* kind, const int64_t* index,
                     const int64_t* variable, const double* value, const double* value2, int64_t presolved_rows,
                     const int64_t* row_map, int64_t presolved_cols, const int64_t* col_map,
                     const double* reduced_primal, int64_t reduced_cols, const double* reduced_dual,
                     int64_t reduced_rows, double* primal, double* dual, double* objective);

#ifdef __cplusplus
}
#endif

#endif
