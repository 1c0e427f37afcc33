// Per-iteration kernels of the PDHG loop (src/lp/first_order/pdlp.cpp:194-262).
//
// Every SpMV is fused with the vector update that consumes it, so one
// iteration is two passes over the matrix: CSC (A^T y, the primal step) and
// CSR (A x-bar, the dual step).  G lanes cooperate on one column/row ("vector
// per row"; G = 32 is warp per row), chosen by the host from the mean line
// length.  T is the storage/arithmetic type of the matrix and iterates
// (double for the FP64 engine, float for the FP32 engine); every reduction
// that feeds a decision (step size, KKT, restart) accumulates in double.
#pragma once

#include "common.cuh"

namespace mc {

// Pointers and sizes of one device-resident problem.
template <class T>
struct Iterates {
    int m, n;
    const int* csc_start;   // [n+1]
    const int* csc_row;     // [nnz]
    const T* csc_val;       // [nnz] scaled A, column major
    const int* csr_start;   // [m+1]
    const int* csr_col;     // [nnz]
    const T* csr_val;       // [nnz] scaled A, row major
    const T* c;             // [n] scaled objective (minimisation sign)
    const T* lo;            // [n] scaled bounds, +-1e300 sentinels
    const T* hi;
    const T* blo;           // [m] scaled row bounds
    const T* bhi;
    const T* col_norm;      // [n] L1 norms of the scaled columns
    const T* row_norm;      // [m]
    T* x;                   // [n]
    T* x_bar;               // [n]
    T* x_avg;               // [n]
    T* dx;                  // [n] staged kernels' scratch
    T* xdx;                 // [2n] (x-bar_j, dx_j) pairs, written on step-size iterations
                            //      for the probe (16-byte aligned)
    T* y;                   // [m]
    T* y_avg;               // [m]
    T* ax_bar;              // [m] step-size iterations only
    double* partials;       // [NUM_SLOTS * kMaxPartials]
    DevState* st;
};

// Original-space data used by the residual pass (pdlp.cpp:62-135).
struct Original {
    const double* c;        // obj_sign * objective, unscaled
    const double* obj;      // objective as given (primal objective :113-115)
    const double* lo;       // variable bounds, sentinel form
    const double* hi;
    const double* blo;      // row bounds, sentinel form
    const double* bhi;
    const double* col_scale;
    const double* row_scale;
    double offset;
};

struct Controls {
    double primal_tol, dual_tol, gap_tol;
    double restart_reduction;
    double weight_smoothing;
    long long restart_every;
    int strategy;          // 0 none, 1 adaptive, 2 fixed
    int adaptive_step;
    int adaptive_weight;
};

template <class T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
template <class T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <class T> __device__ __forceinline__ T sub_rn(T a, T b);
template <> __device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
template <class T> __device__ __forceinline__ T div_rn(T a, T b);
template <> __device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
template <> __device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// Dot of line `j` of a compressed matrix with vector v, G lanes per line,
// four independent gathers in flight per lane per step.  The matrix is
// streamed (evict-first); v is gathered with the keep policy.
// (Loading the matrix in aligned 16-byte quads per lane instead was measured
// on B200 at the 40M-nonzero LP: no faster -- 0.248 / 0.245 ms per primal /
// dual launch against 0.244 / 0.245 -- as the streamed lines already merge in
// L1 between a lane group's unrolled loads.)
template <int G, class T>
__device__ __forceinline__ T line_dot(const int* __restrict__ start, const int* __restrict__ idx,
                                      const T* __restrict__ val, const T* __restrict__ v, int j,
                                      bool valid, int sub, unsigned long long pol) {
    T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
    if (valid) {
        const int b = __ldg(start + j), e = __ldg(start + j + 1);
        int p = b + sub;
        for (; p + 3 * G < e; p += 4 * G) {
            const int i0 = ld_stream(idx + p), i1 = ld_stream(idx + p + G);
            const int i2 = ld_stream(idx + p + 2 * G), i3 = ld_stream(idx + p + 3 * G);
            const T a0 = ld_stream(val + p), a1 = ld_stream(val + p + G);
            const T a2 = ld_stream(val + p + 2 * G), a3 = ld_stream(val + p + 3 * G);
            s0 = fma(a0, ld_keep(v + i0, pol), s0);
            s1 = fma(a1, ld_keep(v + i1, pol), s1);
            s2 = fma(a2, ld_keep(v + i2, pol), s2);
            s3 = fma(a3, ld_keep(v + i3, pol), s3);
        }
        for (; p < e; p += G) s0 = fma(ld_stream(val + p), ld_keep(v + ld_stream(idx + p), pol), s0);
    }
    return group_sum<G>((s0 + s1) + (s2 + s3));
}

// Two dots of the same line against an interleaved pair vector vw[2c] = v_c,
// vw[2c+1] = w_c (A x-bar and A dx on step-size iterations): one gather per
// entry brings both, two entries per lane per step.
template <int G, class T>
__device__ __forceinline__ void line_dot2(const int* __restrict__ start, const int* __restrict__ idx,
                                          const T* __restrict__ val, const T* __restrict__ vw, int j,
                                          bool valid, int sub, T& out_v, T& out_w, unsigned long long pol) {
    T sv0 = T(0), sw0 = T(0), sv1 = T(0), sw1 = T(0);
    if (valid) {
        const int b = __ldg(start + j), e = __ldg(start + j + 1);
        int p = b + sub;
        for (; p + G < e; p += 2 * G) {
            const int i0 = ld_stream(idx + p), i1 = ld_stream(idx + p + G);
            const T a0 = ld_stream(val + p), a1 = ld_stream(val + p + G);
            T v0, w0, v1, w1;
            ld_keep2(vw + 2LL * i0, pol, v0, w0);
            ld_keep2(vw + 2LL * i1, pol, v1, w1);
            sv0 = fma(a0, v0, sv0);
            sw0 = fma(a0, w0, sw0);
            sv1 = fma(a1, v1, sv1);
            sw1 = fma(a1, w1, sw1);
        }
        if (p < e) {
            const int i0 = ld_stream(idx + p);
            const T a0 = ld_stream(val + p);
            T v0, w0;
            ld_keep2(vw + 2LL * i0, pol, v0, w0);
            sv0 = fma(a0, v0, sv0);
            sw0 = fma(a0, w0, sw0);
        }
    }
    out_v = group_sum<G>(sv0 + sv1);
    out_w = group_sum<G>(sw0 + sw1);
}

// Plain y = A x over a compressed-row matrix (kernel-level entry point).
template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_spmv(int rows, const int* __restrict__ start,
                                                 const int* __restrict__ idx, const T* __restrict__ val,
                                                 const T* __restrict__ x, T* __restrict__ y) {
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long pol = policy_keep();
    for (long long t = warp; t * LPW < rows; t += nwarps) {
        const int i = (int)(t * LPW) + slot;
        const bool valid = i < rows;
        const T s = line_dot<G>(start, idx, val, x, i, valid, sub, pol);
        if (valid && sub == 0) y[i] = s;
    }
}

// ------------------------------------------------------------------ primal
// g = c + A^T y; x+ = clamp(x - tau g, l, u); x-bar = 2x+ - x; x_avg update;
// on step-size iterations also dx and sum col_norm dx^2  (pdlp.cpp:195-206, :226)
template <int G, bool STEP, class T>
__global__ void __launch_bounds__(kBlock) k_primal(Iterates<T> P, int k) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    const T step = T(st->eta / st->omega);          // tau_j = (eta/omega)/col_norm_j (:182)
    const T cnt = T((double)(st->avg_count + k + 1));
    constexpr int LPW = 32 / G;                      // lines per warp
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    for (long long t = warp; t * LPW < P.n; t += nwarps) {
        const int j = (int)(t * LPW) + slot;
        const bool valid = j < P.n;
        const bool owner = valid && sub == 0;
        // the line's own vector entries are loaded before the SpMV so that
        // their latency overlaps the matrix stream and the gathers
        T cn = T(1), cj = T(0), xo = T(0), lj = T(0), hj = T(0), xa = T(0);
        if (owner) {
            cn = ld_stream(P.col_norm + j);
            cj = ld_stream(P.c + j);
            xo = ld_stream(P.x + j);
            lj = ld_stream(P.lo + j);
            hj = ld_stream(P.hi + j);
            xa = ld_stream(P.x_avg + j);
        }
        const T aty = line_dot<G>(P.csc_start, P.csc_row, P.csc_val, P.y, j, valid, sub, pol);
        if (owner) {
            const T g = add_rn(cj, aty);
            const T tau = div_rn(step, cn);
            const T xp = clampv(sub_rn(xo, mul_rn(tau, g)), lj, hj);
            const T d = sub_rn(xp, xo);
            const T xb = sub_rn(mul_rn(T(2), xp), xo);
            if (STEP) {  // the probe reads x-bar and dx as pairs; x-bar alone is not read
                st_keep2(P.xdx + 2LL * j, xb, d, pol);
                acc += __dmul_rn(__dmul_rn((double)cn, (double)d), (double)d);
            } else {
                st_keep(P.x_bar + j, xb, pol);
            }
            st_stream(P.x + j, xp);
            st_stream(P.x_avg + j, add_rn(xa, div_rn(sub_rn(xp, xa), cnt)));
        }
    }
    if (STEP) {
        acc = block_reduce(acc, scratch, OpSum());
        if (threadIdx.x == 0) P.partials[SLOT_DX * kMaxPartials + blockIdx.x] = acc;
    }
}

// ------------------------------------------------------------------- dual
// v = y + sigma (A x-bar); y+ = v - sigma clamp(v/sigma, b_lo, b_hi); y_avg
// (pdlp.cpp:220-224, :227)
// The row's own vector entries, loaded ahead of the SpMV.
template <class T>
struct RowData {
    T rn, yo, bl, bh, ya;
};
template <class T>
__device__ __forceinline__ RowData<T> load_row(const Iterates<T>& P, int i) {
    return RowData<T>{ld_stream(P.row_norm + i), ld_stream(P.y + i), ld_stream(P.blo + i), ld_stream(P.bhi + i),
                      ld_stream(P.y_avg + i)};
}
template <class T>
__device__ __forceinline__ void dual_update(const Iterates<T>& P, int i, const RowData<T>& r, T ax, T sg, T cnt,
                                            unsigned long long pol) {
    const T sigma = div_rn(sg, r.rn);
    const T v = add_rn(r.yo, mul_rn(sigma, ax));
    const T yn = sub_rn(v, mul_rn(sigma, clampv(div_rn(v, sigma), r.bl, r.bh)));
    st_keep(P.y + i, yn, pol);
    st_stream(P.y_avg + i, add_rn(r.ya, div_rn(sub_rn(yn, r.ya), cnt)));
}
template <class T>
__device__ __forceinline__ void dual_update(const Iterates<T>& P, int i, T ax, T sg, T cnt,
                                            unsigned long long pol) {
    dual_update(P, i, load_row(P, i), ax, sg, cnt, pol);
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_dual(Iterates<T> P, int k) {
    const DevState* st = P.st;
    if (st->done) return;
    const T sg = T(st->eta * st->omega);             // sigma_i = (eta*omega)/row_norm_i (:183)
    const T cnt = T((double)(st->avg_count + k + 1));
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long pol = policy_keep();
    for (long long t = warp; t * LPW < P.m; t += nwarps) {
        const int i = (int)(t * LPW) + slot;
        const bool valid = i < P.m;
        RowData<T> r{};
        if (valid && sub == 0) r = load_row(P, i);
        const T ax = line_dot<G>(P.csr_start, P.csr_col, P.csr_val, P.x_bar, i, valid, sub, pol);
        if (valid && sub == 0) dual_update(P, i, r, ax, sg, cnt, pol);
    }
}

// Step-size iteration, part 1: A x-bar (kept) and A dx -> sum (A dx)_i^2 / row_norm_i
// (pdlp.cpp:207-210, :220).  The dual update waits for the new eta.
template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_dual_probe(Iterates<T> P) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    for (long long t = warp; t * LPW < P.m; t += nwarps) {
        const int i = (int)(t * LPW) + slot;
        const bool valid = i < P.m;
        T axb, adx;
        line_dot2<G>(P.csr_start, P.csr_col, P.csr_val, P.xdx, i, valid, sub, axb, adx, pol);
        if (valid && sub == 0) {
            P.ax_bar[i] = axb;
            const double a = (double)adx;
            acc += __ddiv_rn(__dmul_rn(a, a), (double)P.row_norm[i]);
        }
    }
    acc = block_reduce(acc, scratch, OpSum());
    if (threadIdx.x == 0) P.partials[SLOT_ADX * kMaxPartials + blockIdx.x] = acc;
}

// Step-size iteration, part 2: the adaptive eta rule (pdlp.cpp:207-219).
__global__ void k_step_size(double* __restrict__ partials, int nprimal, int ndual, DevState* __restrict__ st,
                            Controls ctl) {
    __shared__ double scratch[32];
    if (st->done) return;
    const double dx_norm_sq = reduce_partials(partials + SLOT_DX * kMaxPartials, nprimal, scratch, OpSum());
    const double adx_norm_sq = reduce_partials(partials + SLOT_ADX * kMaxPartials, ndual, scratch, OpSum());
    if (threadIdx.x == 0 && ctl.adaptive_step && dx_norm_sq > 1e-14 && adx_norm_sq > 1e-14) {
        const double L = sqrt(adx_norm_sq / dx_norm_sq);
        if (L > 1e-6) {
            const double target = 0.95 / L;
            const double eta = st->eta;
            if (target < eta) st->eta = maxv(0.1, maxv(target, eta * 0.8));
            else if (target > 1.05 * eta && eta < 0.99) st->eta = minv(0.99, eta * 1.05);
        }
    }
}

// Step-size iteration, part 3: the dual update from the kept A x-bar.
template <class T>
__global__ void __launch_bounds__(kBlock) k_dual_apply(Iterates<T> P, int k) {
    const DevState* st = P.st;
    if (st->done) return;
    const T sg = T(st->eta * st->omega);
    const T cnt = T((double)(st->avg_count + k + 1));
    const unsigned long long pol = policy_keep();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.m; i += gridDim.x * blockDim.x)
        dual_update(P, i, P.ax_bar[i], sg, cnt, pol);
}

// --------------------------------------------------------------- residuals
// compute_unscaled_residuals (pdlp.cpp:62-135) over the averages.  The row and
// column terms are shared by the FP64 kernels below and the mixed-precision
// kernels (mixed.cuh), which evaluate the same formulas on base + correction.

// Row i: s = (A x_avg)_i in the scaled space, y_avg_i scaled.
struct RowTerms {
    double vmax = 0.0, dsum = 0.0, bad = 0.0;
    __device__ __forceinline__ void add(const Original& O, int i, double s, double y_scaled) {
        const double ax = __ddiv_rn(s, O.row_scale[i]);
        const double lo = O.blo[i], hi = O.bhi[i];
        const double proj = clampv(ax, lo, hi);
        const double r = fabs(ax - proj);
        const double sc = 1.0 + maxv(fabs(ax), fabs(proj) < 1e299 ? fabs(proj) : 0.0);
        vmax = maxv(vmax, r / sc);
        const double yu = __dmul_rn(y_scaled, O.row_scale[i]);
        if (yu > 0.0 && hi < 1e299) dsum -= __dmul_rn(yu, hi);
        else if (yu < 0.0 && lo > -1e299) dsum -= __dmul_rn(yu, lo);
        if (!isfinite(ax) || !isfinite(yu)) bad += 1.0;
    }
    __device__ __forceinline__ void store(double* partials, double* scratch) {
        vmax = block_reduce(vmax, scratch, OpMax());
        if (threadIdx.x == 0) partials[SLOT_ROW_MAX * kMaxPartials + blockIdx.x] = vmax;
        dsum = block_reduce(dsum, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_ROW_DOBJ * kMaxPartials + blockIdx.x] = dsum;
        bad = block_reduce(bad, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_NAN * kMaxPartials + blockIdx.x] = bad;
    }
};

// Column j: s = (A^T y_avg)_j in the scaled space, x_avg_j scaled.
struct ColTerms {
    double vmax = 0.0, dres = 0.0, pobj = 0.0, dobj = 0.0, bad = 0.0;
    __device__ __forceinline__ void add(const Original& O, int j, double s, double x_scaled) {
        add_b(O, j, s, x_scaled, O.lo[j], O.hi[j]);
    }
    // the same with the column's (original, sentinel-form) bounds given
    __device__ __forceinline__ void add_b(const Original& O, int j, double s, double x_scaled, double lo,
                                          double hi) {
        const double aty = __ddiv_rn(s, O.col_scale[j]);
        const double xu = __dmul_rn(x_scaled, O.col_scale[j]);
        const double proj = clampv(xu, lo, hi);
        const double r = fabs(xu - proj);
        const double sc = 1.0 + maxv(fabs(xu), fabs(proj) < 1e299 ? fabs(proj) : 0.0);
        vmax = maxv(vmax, r / sc);
        const double g = __dadd_rn(O.c[j], aty);
        const double xp = clampv(__dsub_rn(xu, g), lo, hi);
        const double diff = __dsub_rn(xu, xp);
        dres += __dmul_rn(diff, diff);
        pobj += __dmul_rn(O.obj[j], xu);
        if (g > 0.0 && lo > -1e299) dobj += __dmul_rn(g, lo);
        else if (g < 0.0 && hi < 1e299) dobj += __dmul_rn(g, hi);
        if (!isfinite(xu) || !isfinite(g)) bad += 1.0;
    }
    __device__ __forceinline__ void store(double* partials, double* scratch) {
        vmax = block_reduce(vmax, scratch, OpMax());
        if (threadIdx.x == 0) partials[SLOT_COL_MAX * kMaxPartials + blockIdx.x] = vmax;
        dres = block_reduce(dres, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_COL_DRES * kMaxPartials + blockIdx.x] = dres;
        pobj = block_reduce(pobj, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_COL_POBJ * kMaxPartials + blockIdx.x] = pobj;
        dobj = block_reduce(dobj, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_COL_DOBJ * kMaxPartials + blockIdx.x] = dobj;
        bad = block_reduce(bad, scratch, OpSum());
        if (threadIdx.x == 0) partials[SLOT_NAN * kMaxPartials + kMaxPartials / 2 + blockIdx.x] = bad;
    }
};

// Row part: (A x_avg)_i unscaled, relative row violation (max), row part of
// the dual objective (sum).
template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_residual_rows(Iterates<T> P, Original O) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    RowTerms acc;
    for (long long t = warp; t * LPW < P.m; t += nwarps) {
        const int i = (int)(t * LPW) + slot;
        const bool valid = i < P.m;
        double s = 0.0;
        if (valid) {
            const int b = P.csr_start[i], e = P.csr_start[i + 1];
            for (int p = b + sub; p < e; p += G)
                s = fma((double)P.csr_val[p], (double)P.x_avg[P.csr_col[p]], s);
        }
        s = group_sum<G>(s);
        if (valid && sub == 0) acc.add(O, i, s, (double)P.y_avg[i]);
    }
    acc.store(P.partials, scratch);
}

// Column part: (A^T y_avg)_j unscaled, bound violation (max), squared dual
// residual (sum), primal objective (sum), column part of the dual objective.
template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_residual_cols(Iterates<T> P, Original O) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    ColTerms acc;
    for (long long t = warp; t * LPW < P.n; t += nwarps) {
        const int j = (int)(t * LPW) + slot;
        const bool valid = j < P.n;
        double s = 0.0;
        if (valid) {
            const int b = P.csc_start[j], e = P.csc_start[j + 1];
            for (int p = b + sub; p < e; p += G)
                s = fma((double)P.csc_val[p], (double)P.y_avg[P.csc_row[p]], s);
        }
        s = group_sum<G>(s);
        if (valid && sub == 0) acc.add(O, j, s, (double)P.x_avg[j]);
    }
    acc.store(P.partials, scratch);
}

// Device trace of the restart checks (optional).
struct TraceBuf {
    long long capacity;
    long long* iteration;
    double* primal;
    double* dual;
    double* gap;
    double* eta;
    double* omega;
    int* restarted;
};

// Restart check (pdlp.cpp:229-261): KKT scalars, termination, adaptive
// restart, primal weight.  `span` = iterations in the chunk just finished;
// `final_pass` = evaluate only (loop exhausted, :263-275).
__global__ void k_finalize(double* __restrict__ partials, int nrow_parts, int ncol_parts, long long span,
                           int final_pass, double offset, Controls ctl, TraceBuf tr,
                           DevState* __restrict__ st) {
    __shared__ double scratch[32];
    if (st->done) return;
    const double row_max = reduce_partials(partials + SLOT_ROW_MAX * kMaxPartials, nrow_parts, scratch, OpMax());
    const double row_dobj = reduce_partials(partials + SLOT_ROW_DOBJ * kMaxPartials, nrow_parts, scratch, OpSum());
    const double col_max = reduce_partials(partials + SLOT_COL_MAX * kMaxPartials, ncol_parts, scratch, OpMax());
    const double col_dres = reduce_partials(partials + SLOT_COL_DRES * kMaxPartials, ncol_parts, scratch, OpSum());
    const double col_pobj = reduce_partials(partials + SLOT_COL_POBJ * kMaxPartials, ncol_parts, scratch, OpSum());
    const double col_dobj = reduce_partials(partials + SLOT_COL_DOBJ * kMaxPartials, ncol_parts, scratch, OpSum());
    const double bad_rows = reduce_partials(partials + SLOT_NAN * kMaxPartials, nrow_parts, scratch, OpSum());
    const double bad_cols = reduce_partials(partials + SLOT_NAN * kMaxPartials + kMaxPartials / 2, ncol_parts,
                                            scratch, OpSum());
    if (threadIdx.x != 0) return;
    const double primal = maxv(row_max, col_max);
    const double dual = sqrt(col_dres) / st->c_scale;
    const double pobj = offset + col_pobj;
    const double dobj = (offset + row_dobj) + col_dobj;
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double score = maxv(maxv(primal, dual), gap);
    st->primal_infeas = primal;
    st->dual_infeas = dual;
    st->gap = gap;
    st->objective = pobj;
    st->dual_objective = dobj;
    st->score = score;
    st->restart_pending = 0;
    const long long iter = st->iter + span;
    const long long isr = st->iters_since_restart + span;
    int restarted = 0;
    if (bad_rows + bad_cols > 0.0 || !isfinite(score)) {
        // non-finite iterates: numerical_failure (the reference would run on to
        // its iteration limit on NaNs; stopping is the engine's extension)
        st->nonfinite = 1;
        st->done = 1;
        st->status = 3;
    } else if (!final_pass && primal <= ctl.primal_tol && dual <= ctl.dual_tol && gap <= ctl.gap_tol) {
        st->done = 1;
        st->status = 0;
    } else if (!final_pass) {
        const bool do_restart =
            ctl.strategy == 2 ||
            (ctl.strategy == 1 && (score <= ctl.restart_reduction * st->last_restart_score ||
                                   (isr >= 5 * ctl.restart_every && score < st->last_restart_score)));
        if (do_restart) {
            if (ctl.adaptive_weight && primal > 1e-12 && dual > 1e-12) {
                const double ratio = clampv(sqrt(primal / dual), 0.05, 20.0);
                st->omega = clampv(st->omega * pow(ratio, ctl.weight_smoothing), 1e-6, 1e6);
            }
            st->restart_pending = 1;
            st->avg_count = 0;
            st->iters_since_restart = 0;
            st->last_restart_score = score;
            st->restarts += 1;
            restarted = 1;
        } else {
            st->avg_count += span;
            st->iters_since_restart = isr;
        }
    }
    st->iter = iter;
    if (tr.capacity > 0 && st->checks < tr.capacity && !final_pass) {
        const long long q = st->checks;
        tr.iteration[q] = iter;
        tr.primal[q] = primal;
        tr.dual[q] = dual;
        tr.gap[q] = gap;
        tr.eta[q] = st->eta;
        tr.omega[q] = st->omega;
        tr.restarted[q] = restarted;
    }
    if (!final_pass) st->checks += 1;
}

// Restart to the average (pdlp.cpp:257-258): x <- x_avg, y <- y_avg.
template <class T>
__global__ void __launch_bounds__(kBlock) k_restart_copy(Iterates<T> P) {
    const DevState* st = P.st;
    if (!st->restart_pending || st->done) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n + P.m; t += gridDim.x * blockDim.x) {
        if (t < P.n) P.x[t] = P.x_avg[t];
        else P.y[t - P.n] = P.y_avg[t - P.n];
    }
}

}  // namespace mc
