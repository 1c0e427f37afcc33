/*
 * Seeded synthetic LP generators for the PDLP engine's workloads.
 *
 * Every generator is a pure function of its seed: splitmix64 for the raw
 * stream, Box-Muller for normals (std::normal_distribution is
 * implementation-defined, so it is not used anywhere).  The caller allocates
 * every output array (sizes are stated per function) and the generator fills
 * them, so Python/numpy, C and C++ callers share one code path.
 *
 * Matrix layout: CSC with int32 column pointers and row indices, rows strictly
 * increasing inside each column -- the input layout of the reference model
 * (include/markov_cero/model/model.hpp:25-34) with 32-bit indices.
 * Infinite bounds are +-INFINITY.
 */
#ifndef MC_LPGEN_H
#define MC_LPGEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Random-LP families. */
enum {
    LPGEN_STANDARD = 0,  /* N(0,1) values, 0 <= x <= 10, equality rows        */
    LPGEN_PRECISION = 1  /* |a| log-uniform [1e-3,1e3], random sign, 20% of
                            columns boxed by u~U(1,100), the rest x >= 0      */
};

/*
 * Random LP with a known optimum.
 *   A: m x n, exactly k nonzeros per column at distinct uniform rows.
 *   x*: 70% of columns U(0.1,5), 30% at 0.   y* ~ N(0,1).
 *   s: 0 on interior columns, U(0.1,2) on columns at 0; in the PRECISION
 *      family a boxed column whose drawn x* exceeds u is set to x* = u with
 *      s = -U(0.1,2) (an active upper bound).
 *   b = A x* (rows are equalities), c = A^T y* + s, minimise c^T x.
 * Outputs (caller-allocated):
 *   col_start[n+1], row_index[n*k], value[n*k], objective[n], var_lower[n],
 *   var_upper[n], row_lower[m], row_upper[m], x_star[n], y_star[m];
 *   opt[0] = c.x* and opt[1] = b.y* (both accumulated in long double).
 * Returns 0, or -1 on bad sizes (k > m, k < 1, n*k >= 2^31).
 */
int lpgen_random_lp(uint64_t seed, int32_t m, int32_t n, int32_t k, int32_t family,
                    int32_t* col_start, int32_t* row_index, double* value,
                    double* objective, double* var_lower, double* var_upper,
                    double* row_lower, double* row_upper,
                    double* x_star, double* y_star, double* opt);

/*
 * Transportation LP: S suppliers, D customers, points uniform in the unit
 * square, cost_sd = |p_s - p_d| * (1 + 0.1 N(0,1)) clipped at 0,
 * supply = Dirichlet(1) * 1100 (rows <=), demand = Dirichlet(1) * 1000
 * (rows =), x >= 0.  Column j = s*D + d has rows s and S+d (value 1).
 * m = S+D, n = S*D, nnz = 2*S*D.
 * Outputs: col_start[n+1], row_index[2n], value[2n], objective[n],
 * var_lower[n], var_upper[n], row_lower[m], row_upper[m];
 * features (optional, may be NULL): sup_xy[2S], dem_xy[2D] point coordinates.
 */
int lpgen_transport(uint64_t seed, int32_t S, int32_t D,
                    int32_t* col_start, int32_t* row_index, double* value,
                    double* objective, double* var_lower, double* var_upper,
                    double* row_lower, double* row_upper,
                    double* sup_xy, double* dem_xy);

/* Draws used by the batch workloads, exposed so every caller agrees:
 * uniform integer in [lo, hi] from stream (seed, index). */
int64_t lpgen_uniform_int(uint64_t seed, uint64_t index, int64_t lo, int64_t hi);
double lpgen_uniform01(uint64_t seed, uint64_t index);

/*
 * Node-variant bound tightening in the style of branch-and-bound children:
 * from base bounds (lo, hi) and the base optimum x*, tighten `count` random
 * distinct columns (count ~ U{1..10}) to floor or ceil of x*_j +- U(0,1):
 * with probability 1/2 the upper bound becomes floor(x*_j - U), otherwise the
 * lower bound becomes ceil(x*_j + U).  lo/hi are updated in place.  A bound
 * may cross the other one, which makes the variant infeasible on purpose.
 * Returns the number of tightened columns, or -1 on bad sizes.
 */
int lpgen_tighten_bounds(uint64_t seed, int32_t n, const double* x_star,
                         double* var_lower, double* var_upper,
                         int32_t* tightened_columns /* [10], may be NULL */);

#ifdef __cplusplus
}
#endif

#endif
