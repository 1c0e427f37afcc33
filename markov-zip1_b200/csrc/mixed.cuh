// Mixed-precision PDHG (MC_PRECISION_FP32_REFINE).
//
// The iterate is held as an FP64 base plus an FP32 correction,
//     x = x_hat + dx,   y = y_hat + dy      (equilibrated space),
// and the FP32 kernels iterate on the correction LP
//     min  g_hat' dx   s.t.  lo - x_hat <= dx <= hi - x_hat,
//          rows: b_lo - A x_hat <= A dx <= b_hi - A x_hat,
//     g_hat = c + A^T y_hat (the reduced costs at the base),
// which PDHG follows exactly as it would the original LP (the primal prox is
// translation-equivariant; the dual prox is rewritten below so that only the
// FP64-computed residuals A x_hat - b enter it).  The matrix, the gathered
// vectors and every per-line vector are FP32, so one iteration moves about
// 16 bytes per nonzero instead of 24.
//
// Everything that decides -- the KKT residuals, the duality gap, the restart
// test and the primal weight -- is evaluated in FP64 on x_hat + dx_avg with
// the FP64 copy of A, by the reference's definition (pdlp.cpp:62-135).  At
// every restart to the average the base moves there (x_hat += dx_avg), the
// correction restarts from zero, and the correction LP's data are recomputed
// in FP64 from the same FP64 SpMVs the residual pass just did: each restart
// is an iterative-refinement step that re-solves the residual LP from the
// current point, so FP32 rounding never accumulates beyond one restart cycle.
#pragma once

#include "common.cuh"
#include "iter_kernels.cuh"

namespace mc {

// FP64 base and the per-cycle FP32 data of the correction LP.
struct MixedState {
    double* x_hat;         // [n] base primal (scaled)
    double* y_hat;         // [m] base dual (scaled)
    double* ax_full;       // [m] A (x_hat + dx_avg), written by the residual pass
    double* aty_full;      // [n] A^T (y_hat + dy_avg)
    const double* c64;     // [n] scaled c (FP64)
    const double* lo64;    // [n] scaled bounds, sentinel form
    const double* hi64;
    const double* blo64;   // [m]
    const double* bhi64;
    const double* csc_val64;  // FP64 scaled matrix (residual pass)
    const double* csr_val64;
    float* g;              // [n] float(c + A^T y_hat)       (= Iterates<float>::c)
    float* lo;             // [n] float(lo - x_hat), -inf if unbounded
    float* hi;             // [n]
    float* r_lo;           // [m] float(A x_hat - b_lo), +inf if unbounded
    float* r_hi;           // [m] float(A x_hat - b_hi), -inf if unbounded
    float* yb;             // [m] float(y_hat)
};

// Dual step on the correction (pdlp.cpp:221-224 rewritten):
//   t = (y_hat + dy)/sigma + (A x_hat - b) + A dx_bar  is v/sigma - b;
//   below b_lo:  dy' = dy + sigma (r_lo + A dx_bar)
//   above b_hi:  dy' = dy + sigma (r_hi + A dx_bar)
//   inside:      y' = 0, i.e. dy' = -y_hat
__device__ __forceinline__ void dual_update_mx(const Iterates<float>& P, const MixedState& M, int i, float ax,
                                               float sg, float cnt, unsigned long long pol, float rn, float dy,
                                               float dya, float yb, float rl, float rh) {
    const float sigma = __fdiv_rn(sg, rn);
    const float base = __fdiv_rn(__fadd_rn(yb, dy), sigma);
    float dyn;
    if (__fadd_rn(base, __fadd_rn(rl, ax)) < 0.f) dyn = __fadd_rn(dy, __fmul_rn(sigma, __fadd_rn(rl, ax)));
    else if (__fadd_rn(base, __fadd_rn(rh, ax)) > 0.f) dyn = __fadd_rn(dy, __fmul_rn(sigma, __fadd_rn(rh, ax)));
    else dyn = -yb;
    st_keep(P.y + i, dyn, pol);
    st_stream(P.y_avg + i, __fadd_rn(dya, __fdiv_rn(__fsub_rn(dyn, dya), cnt)));
}

template <int G>
__global__ void __launch_bounds__(kBlock, kMixedRowBlocks) k_dual_mx(Iterates<float> P, MixedState M, int k) {
    const DevState* st = P.st;
    if (st->done) return;
    const float sg = (float)(st->eta * st->omega);
    const float cnt = (float)(double)(st->avg_count + k + 1);
    constexpr int LPW = 32 / G;
    const int lane = threadIdx.x & 31, sub = lane % G, slot = lane / G;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long pol = policy_keep();
    for (long long t = warp; t * LPW < P.m; t += nwarps) {
        const int i = (int)(t * LPW) + slot;
        const bool valid = i < P.m;
        const bool owner = valid && sub == 0;
        float rn = 1.f, dy = 0.f, dya = 0.f, yb = 0.f, rl = 0.f, rh = 0.f;
        if (owner) {
            rn = ld_stream(P.row_norm + i);
            dy = ld_stream(P.y + i);
            dya = ld_stream(P.y_avg + i);
            yb = ld_stream(M.yb + i);
            rl = ld_stream(M.r_lo + i);
            rh = ld_stream(M.r_hi + i);
        }
        const float ax = line_dot<G>(P.csr_start, P.csr_col, P.csr_val, P.x_bar, i, valid, sub, pol);
        if (owner) dual_update_mx(P, M, i, ax, sg, cnt, pol, rn, dy, dya, yb, rl, rh);
    }
}

// Step-size iteration, part 3 for the correction (A dx_bar kept by the probe).
__global__ void __launch_bounds__(kBlock) k_dual_apply_mx(Iterates<float> P, MixedState M, int k) {
    const DevState* st = P.st;
    if (st->done) return;
    const float sg = (float)(st->eta * st->omega);
    const float cnt = (float)(double)(st->avg_count + k + 1);
    const unsigned long long pol = policy_keep();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.m; i += gridDim.x * blockDim.x)
        dual_update_mx(P, M, i, P.ax_bar[i], sg, cnt, pol, ld_stream(P.row_norm + i), ld_stream(P.y + i),
                       ld_stream(P.y_avg + i), ld_stream(M.yb + i), ld_stream(M.r_lo + i), ld_stream(M.r_hi + i));
}

// FP64 residual pass on x_hat + dx_avg, y_hat + dy_avg (FP64 matrix).  Also
// keeps A x and A^T y of that point for the recentring.
template <int G>
__global__ void __launch_bounds__(kBlock) k_residual_rows_mx(Iterates<float> P, MixedState M, Original O) {
    __shared__ double scratch[32];
    if (P.st->done) return;
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
            for (int p = b + sub; p < e; p += G) {
                const int jj = P.csr_col[p];
                s = fma(M.csr_val64[p], M.x_hat[jj] + (double)P.x_avg[jj], s);
            }
        }
        s = group_sum<G>(s);
        if (valid && sub == 0) {
            M.ax_full[i] = s;
            acc.add(O, i, s, M.y_hat[i] + (double)P.y_avg[i]);
        }
    }
    acc.store(P.partials, scratch);
}

template <int G>
__global__ void __launch_bounds__(kBlock) k_residual_cols_mx(Iterates<float> P, MixedState M, Original O) {
    __shared__ double scratch[32];
    if (P.st->done) return;
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
            for (int p = b + sub; p < e; p += G) {
                const int ii = P.csc_row[p];
                s = fma(M.csc_val64[p], M.y_hat[ii] + (double)P.y_avg[ii], s);
            }
        }
        s = group_sum<G>(s);
        if (valid && sub == 0) {
            M.aty_full[j] = s;
            acc.add(O, j, s, M.x_hat[j] + (double)P.x_avg[j]);
        }
    }
    acc.store(P.partials, scratch);
}

// Restart to the average: move the base there and rebuild the correction
// LP's data from the FP64 products of the residual pass.  `force` rebuilds
// unconditionally (the start of a solve, with dx_avg = dy_avg = 0).
__global__ void __launch_bounds__(kBlock) k_recenter_mx(Iterates<float> P, MixedState M, int force) {
    const DevState* st = P.st;
    if (!force && (!st->restart_pending || st->done)) return;
    const float inf = __int_as_float(0x7f800000);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n + P.m; t += gridDim.x * blockDim.x) {
        if (t < P.n) {
            const double xh = M.x_hat[t] + (double)P.x_avg[t];
            M.x_hat[t] = xh;
            P.x[t] = 0.f;
            P.x_avg[t] = 0.f;
            M.g[t] = (float)(M.c64[t] + M.aty_full[t]);
            const double l = M.lo64[t], h = M.hi64[t];
            M.lo[t] = (l <= -1e299) ? -inf : (float)(l - xh);
            M.hi[t] = (h >= 1e299) ? inf : (float)(h - xh);
        } else {
            const int i = t - P.n;
            const double yh = M.y_hat[i] + (double)P.y_avg[i];
            M.y_hat[i] = yh;
            P.y[i] = 0.f;
            P.y_avg[i] = 0.f;
            M.yb[i] = (float)yh;
            const double ax = M.ax_full[i], l = M.blo64[i], h = M.bhi64[i];
            M.r_lo[i] = (l <= -1e299) ? inf : (float)(ax - l);
            M.r_hi[i] = (h >= 1e299) ? -inf : (float)(ax - h);
        }
    }
}

// FP64 -> FP32 copies (matrix values, norms)
__global__ void k_to_float(long long count, const double* __restrict__ in, float* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// Unscaled outputs of the mixed form: x = (x_hat + dx_avg) D_C, y = (y_hat + dy_avg) D_R.
__global__ void k_unscale_out_mx(int n, int m, const double* __restrict__ x_hat, const float* __restrict__ dx_avg,
                                 const double* __restrict__ y_hat, const float* __restrict__ dy_avg,
                                 const double* __restrict__ col_scale, const double* __restrict__ row_scale,
                                 double* __restrict__ x_out, double* __restrict__ y_out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
        if (t < n) {
            if (x_out) x_out[t] = __dmul_rn(x_hat[t] + (double)dx_avg[t], col_scale[t]);
        } else {
            const int i = t - n;
            if (y_out) y_out[i] = __dmul_rn(y_hat[i] + (double)dy_avg[i], row_scale[i]);
        }
    }
}

}  // namespace mc
