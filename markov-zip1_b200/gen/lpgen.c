/*
 * Seeded synthetic LP generators (see lpgen.h for the families).
 *
 * Randomness is counter based: every column, row and variant owns a private
 * splitmix64 stream derived from (seed, purpose, index), so any slice of an
 * instance can be regenerated independently and the columns can be produced
 * in parallel without changing a single bit of the output.
 */
#include "lpgen.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#define LPGEN_PI 3.14159265358979323846

typedef struct { uint64_t s; } rng_t;

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static uint64_t next_u64(rng_t* r) {
    r->s += 0x9E3779B97F4A7C15ULL;
    return mix64(r->s);
}

/* purpose tags keep the per-index streams of different quantities apart */
enum { P_COLUMN = 1, P_ROW = 2, P_VARIANT = 3, P_POINT_S = 4, P_POINT_D = 5, P_MISC = 6 };

static rng_t stream(uint64_t seed, uint64_t purpose, uint64_t index) {
    rng_t r;
    r.s = mix64(mix64(seed + 0x632BE59BD9B4E019ULL) ^ (purpose * 0xD1B54A32D192ED03ULL)) ^
          mix64(index + 0x8CB92BA72F3D8DD7ULL);
    return r;
}

/* uniform in [0,1) with 53 random bits */
static double u01(rng_t* r) { return (double)(next_u64(r) >> 11) * 0x1.0p-53; }
/* uniform in (0,1] */
static double u01_open0(rng_t* r) { return ((double)(next_u64(r) >> 11) + 1.0) * 0x1.0p-53; }
static double uab(rng_t* r, double a, double b) { return a + (b - a) * u01(r); }
/* Box-Muller, one normal per pair of uniforms */
static double normal(rng_t* r) {
    const double u1 = u01_open0(r);
    const double u2 = u01(r);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * LPGEN_PI * u2);
}
static uint32_t below(rng_t* r, uint32_t bound) {
    return (uint32_t)(((unsigned __int128)next_u64(r) * bound) >> 64);
}

int64_t lpgen_uniform_int(uint64_t seed, uint64_t index, int64_t lo, int64_t hi) {
    rng_t r = stream(seed, P_MISC, index);
    if (hi < lo) return lo;
    const uint64_t span = (uint64_t)(hi - lo) + 1ULL;
    return lo + (int64_t)(((unsigned __int128)next_u64(&r) * span) >> 64);
}

double lpgen_uniform01(uint64_t seed, uint64_t index) {
    rng_t r = stream(seed, P_MISC, index ^ 0x5555555555555555ULL);
    return u01(&r);
}

int lpgen_random_lp(uint64_t seed, int32_t m, int32_t n, int32_t k, int32_t family,
                    int32_t* col_start, int32_t* row_index, double* value,
                    double* objective, double* var_lower, double* var_upper,
                    double* row_lower, double* row_upper,
                    double* x_star, double* y_star, double* opt) {
    if (m < 1 || n < 1 || k < 1 || k > m) return -1;
    if ((int64_t)n * (int64_t)k >= (int64_t)1 << 31) return -1;
    if (family != LPGEN_STANDARD && family != LPGEN_PRECISION) return -1;

    /* duals first: one stream per row */
    for (int32_t i = 0; i < m; ++i) {
        rng_t r = stream(seed, P_ROW, (uint64_t)i);
        y_star[i] = normal(&r);
    }

    long double* act = (long double*)calloc((size_t)m, sizeof(long double));
    if (!act) return -2;
    double* s = (double*)malloc((size_t)n * sizeof(double));
    if (!s) { free(act); return -2; }

    col_start[0] = 0;
    for (int32_t j = 0; j < n; ++j) {
        rng_t r = stream(seed, P_COLUMN, (uint64_t)j);
        int32_t* rows = row_index + (int64_t)j * k;
        double* vals = value + (int64_t)j * k;
        /* k distinct rows by rejection, then insertion sort (k <= m) */
        for (int32_t t = 0; t < k; ++t) {
            int32_t cand;
            int dup;
            do {
                cand = (int32_t)below(&r, (uint32_t)m);
                dup = 0;
                for (int32_t q = 0; q < t; ++q) if (rows[q] == cand) { dup = 1; break; }
            } while (dup);
            int32_t p = t;
            while (p > 0 && rows[p - 1] > cand) { rows[p] = rows[p - 1]; --p; }
            rows[p] = cand;
        }
        for (int32_t t = 0; t < k; ++t) {
            if (family == LPGEN_STANDARD) {
                double v = normal(&r);
                if (v == 0.0) v = 1.0; /* the model forbids explicit zeros */
                vals[t] = v;
            } else {
                const double mag = pow(10.0, uab(&r, -3.0, 3.0));
                vals[t] = (next_u64(&r) & 1ULL) ? -mag : mag;
            }
        }
        col_start[j + 1] = (int32_t)((int64_t)(j + 1) * k);

        /* primal optimum, bounds and reduced cost of this column */
        const int interior = u01(&r) < 0.7;
        double xs = interior ? uab(&r, 0.1, 5.0) : 0.0;
        double sj = interior ? 0.0 : uab(&r, 0.1, 2.0);
        double lo = 0.0, hi = 10.0;
        if (family == LPGEN_PRECISION) {
            hi = INFINITY;
            if (u01(&r) < 0.2) {
                hi = uab(&r, 1.0, 100.0);
                if (xs > hi) { xs = hi; sj = -uab(&r, 0.1, 2.0); }
            }
        }
        x_star[j] = xs;
        s[j] = sj;
        var_lower[j] = lo;
        var_upper[j] = hi;
        if (xs != 0.0)
            for (int32_t t = 0; t < k; ++t) act[rows[t]] += (long double)vals[t] * xs;
    }

    long double cx = 0.0L, by = 0.0L, sx = 0.0L;
    for (int32_t i = 0; i < m; ++i) {
        const double b = (double)act[i];
        row_lower[i] = b;
        row_upper[i] = b;
        by += (long double)b * y_star[i];
    }
    for (int32_t j = 0; j < n; ++j) {
        long double g = s[j];
        for (int32_t p = col_start[j]; p < col_start[j + 1]; ++p)
            g += (long double)value[p] * y_star[row_index[p]];
        objective[j] = (double)g;
        cx += (long double)objective[j] * x_star[j];
        sx += (long double)s[j] * x_star[j];
    }
    if (opt) {
        opt[0] = (double)cx;
        opt[1] = (double)(by + sx);
    }
    free(act);
    free(s);
    return 0;
}

int lpgen_transport(uint64_t seed, int32_t S, int32_t D,
                    int32_t* col_start, int32_t* row_index, double* value,
                    double* objective, double* var_lower, double* var_upper,
                    double* row_lower, double* row_upper,
                    double* sup_xy, double* dem_xy) {
    if (S < 1 || D < 1) return -1;
    if ((int64_t)S * D * 2 >= (int64_t)1 << 31) return -1;
    double* ps = (double*)malloc((size_t)S * 2 * sizeof(double));
    double* pd = (double*)malloc((size_t)D * 2 * sizeof(double));
    if (!ps || !pd) { free(ps); free(pd); return -2; }

    /* points and Dirichlet(1) weights (normalised unit exponentials) */
    long double wsum = 0.0L;
    for (int32_t s = 0; s < S; ++s) {
        rng_t r = stream(seed, P_POINT_S, (uint64_t)s);
        ps[2 * s] = u01(&r);
        ps[2 * s + 1] = u01(&r);
        const double e = -log(u01_open0(&r));
        row_upper[s] = e;
        wsum += e;
    }
    for (int32_t s = 0; s < S; ++s) {
        row_upper[s] = (double)((long double)row_upper[s] / wsum * 1100.0L);
        row_lower[s] = -INFINITY;
    }
    long double dsum = 0.0L;
    for (int32_t d = 0; d < D; ++d) {
        rng_t r = stream(seed, P_POINT_D, (uint64_t)d);
        pd[2 * d] = u01(&r);
        pd[2 * d + 1] = u01(&r);
        const double e = -log(u01_open0(&r));
        row_lower[S + d] = e;
        dsum += e;
    }
    for (int32_t d = 0; d < D; ++d) {
        const double dem = (double)((long double)row_lower[S + d] / dsum * 1000.0L);
        row_lower[S + d] = dem;
        row_upper[S + d] = dem;
    }
    col_start[0] = 0;
    for (int32_t s = 0; s < S; ++s) {
        for (int32_t d = 0; d < D; ++d) {
            const int64_t j = (int64_t)s * D + d;
            rng_t r = stream(seed, P_COLUMN, (uint64_t)j);
            const double dx = ps[2 * s] - pd[2 * d];
            const double dy = ps[2 * s + 1] - pd[2 * d + 1];
            double cost = sqrt(dx * dx + dy * dy) * (1.0 + 0.1 * normal(&r));
            if (cost < 0.0) cost = 0.0;
            objective[j] = cost;
            var_lower[j] = 0.0;
            var_upper[j] = INFINITY;
            row_index[2 * j] = s;
            row_index[2 * j + 1] = S + d;
            value[2 * j] = 1.0;
            value[2 * j + 1] = 1.0;
            col_start[j + 1] = (int32_t)(2 * (j + 1));
        }
    }
    if (sup_xy) for (int32_t q = 0; q < 2 * S; ++q) sup_xy[q] = ps[q];
    if (dem_xy) for (int32_t q = 0; q < 2 * D; ++q) dem_xy[q] = pd[q];
    free(ps);
    free(pd);
    return 0;
}

int lpgen_tighten_bounds(uint64_t seed, int32_t n, const double* x_star,
                         double* var_lower, double* var_upper, int32_t* tightened_columns) {
    if (n < 1) return -1;
    rng_t r = stream(seed, P_VARIANT, 0);
    int32_t count = 1 + (int32_t)below(&r, 10u);
    if (count > n) count = n;
    int32_t chosen[10];
    for (int32_t t = 0; t < count; ++t) {
        int32_t cand;
        int dup;
        do {
            cand = (int32_t)below(&r, (uint32_t)n);
            dup = 0;
            for (int32_t q = 0; q < t; ++q) if (chosen[q] == cand) { dup = 1; break; }
        } while (dup);
        chosen[t] = cand;
        const double shift = u01(&r);
        if (next_u64(&r) & 1ULL) {
            const double v = floor(x_star[cand] - shift);
            if (v < var_upper[cand]) var_upper[cand] = v;
        } else {
            const double v = ceil(x_star[cand] + shift);
            if (v > var_lower[cand]) var_lower[cand] = v;
        }
        if (tightened_columns) tightened_columns[t] = cand;
    }
    return count;
}
