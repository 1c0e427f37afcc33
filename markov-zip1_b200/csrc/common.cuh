// Shared device helpers of the PDLP engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace mc {

// The reference encodes infinite bounds as +-1e300 inside the solver
// (src/lp/first_order/pdlp.cpp:47-48, :163-164).
constexpr double kBig = 1e300;
constexpr int kBlock = 256;          // threads per block of the streaming kernels
// Resident blocks per SM asked of the compiler for the FP32 row kernels
// (40 registers, no spills): on B200 the mixed dual SpMV runs 11% faster at 6
// blocks than at the compiler's 48 registers / 5 blocks.  The FP64 kernels
// spill under the same cap and run slower, so they keep the default.
constexpr int kMixedRowBlocks = 6;
constexpr int kMaxPartials = 4096;   // per-slot capacity of the block-partials buffer

// Slots of the block-partials buffer (one double per block per slot).
enum PartialSlot : int {
    SLOT_DX = 0,        // sum col_norm * dx^2               (primal, step-size iterations)
    SLOT_ADX = 1,       // sum (A dx)_i^2 / row_norm_i        (dual, step-size iterations)
    SLOT_ROW_MAX = 2,   // max relative row violation        (residual)
    SLOT_ROW_DOBJ = 3,  // row part of the dual objective    (residual)
    SLOT_COL_MAX = 4,   // max relative bound violation      (residual)
    SLOT_COL_DRES = 5,  // sum of squared dual residuals     (residual)
    SLOT_COL_POBJ = 6,  // primal objective                  (residual)
    SLOT_COL_DOBJ = 7,  // column part of the dual objective (residual)
    SLOT_A = 8,         // setup scratch
    SLOT_B = 9,
    SLOT_C = 10,
    SLOT_NAN = 11,      // count of non-finite values seen in a residual pass
    // batch residual pass: the Farkas test of the dual ray candidate d (batch_kernels.cuh)
    SLOT_RAY_L = 12,       // sum_j (g_j > 0 ? g_j lo_j : g_j hi_j), g = A^T d          (columns)
    SLOT_RAY_CSCALE = 13,  // sum_j |bound_j| sum_i |a_ij d_i|: rounding scale        (columns)
    SLOT_RAY_CINF = 14,    // count of nonzero g_j meeting an infinite bound           (columns)
    SLOT_RAY_RSCALE = 15,  // sum_i |d_i bound_i|                                      (rows)
    SLOT_RAY_RINF = 16,    // count of nonzero d_i meeting an infinite bound           (rows)
    SLOT_RAY_U = 17,       // sum_i (d_i > 0 ? d_i hi_i : d_i lo_i)                    (rows)
    NUM_SLOTS = 18
};

// Scalars of one solve, resident in device memory so that whole restart
// chunks run from a CUDA graph without host round trips.
struct DevState {
    double eta;                 // step size factor (pdlp.cpp:179)
    double omega;               // primal weight (pdlp.cpp:177-178)
    double last_restart_score;  // pdlp.cpp:193
    double primal_infeas, dual_infeas, gap, objective, dual_objective, score;
    double c_norm_inf, b_norm_inf, c_scale;  // c_scale: max(1, |c_orig|_inf) of the residual
    long long iter;                 // iterations completed at the start of the chunk
    long long avg_count;            // averaging count at the start of the chunk
    long long iters_since_restart;  // at the start of the chunk
    long long restarts;
    long long checks;
    long long ruiz_passes;          // scaling passes executed
    int done;                       // 1 once a terminal status is set
    int status;                     // mc_pdlp_status when done
    int restart_pending;            // finalize -> restart copy
    int ruiz_done;                  // Ruiz converged: later passes are no-ops
    int nonfinite;                  // a residual pass saw NaN/Inf
    int active_tiles[2];            // batch poll state: running column / row tiles
    int cert;                       // batch: MC_CERT_* kind when status is infeasible
    int pad[3];
};

// ---- cache policy helpers -------------------------------------------------
// The matrix and the per-line vectors are streamed once per iteration: they
// are loaded with the "streaming" (evict-first) hint so that they do not push
// the gathered iterate (x-bar, 40 MB at 5M columns; y, 16 MB at 2M rows) out
// of L2.  The gathered iterate is written and read with an L2 evict_last
// policy so that it stays resident between the kernel that writes it and the
// kernel that gathers from it.
__device__ __forceinline__ unsigned long long policy_keep() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// The random gathers skip L1 allocation (no reuse there; measured 4-5%
// faster SpMV kernels on B200 than with L1 allocation).
__device__ __forceinline__ double ld_keep(const double* a, unsigned long long pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_keep(const float* a, unsigned long long pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
// One 16-byte (8-byte for float) gather of an interleaved pair: both values
// come from the same sector, so the pair costs one L2 request, not two.
__device__ __forceinline__ void ld_keep2(const double* a, unsigned long long pol, double& u, double& v) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(u), "=d"(v) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void ld_keep2(const float* a, unsigned long long pol, float& u, float& v) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
        : "=f"(u), "=f"(v) : "l"(a), "l"(pol));
}
__device__ __forceinline__ void st_keep2(double* a, double u, double v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(a), "d"(u), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep2(float* a, float u, float v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(a), "f"(u), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep(double* a, double v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_keep(float* a, float v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}
template <class T>
__device__ __forceinline__ T ld_stream(const T* a) { return __ldcs(a); }
template <class T>
__device__ __forceinline__ void st_stream(T* a, T v) { __stcs(a, v); }

// std::clamp(v, lo, hi): lo if v < lo, hi if hi < v, else v.
template <class T>
__device__ __forceinline__ T clampv(T v, T lo, T hi) {
    return (v < lo) ? lo : ((hi < v) ? hi : v);
}
// std::max / std::min (first argument kept on ties)
template <class T>
__device__ __forceinline__ T maxv(T a, T b) { return (a < b) ? b : a; }
template <class T>
__device__ __forceinline__ T minv(T a, T b) { return (b < a) ? b : a; }

// Butterfly sum over aligned groups of G lanes; every lane of the warp must
// call it.  Fixed order, so results are run-to-run deterministic.
template <int G, class T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

struct OpSum {
    __device__ __forceinline__ double operator()(double a, double b) const { return a + b; }
    static constexpr double identity = 0.0;
};
struct OpMax {
    __device__ __forceinline__ double operator()(double a, double b) const { return maxv(a, b); }
    static constexpr double identity = 0.0;  // all maxima here are of non-negative values
};

// Block-wide reduction in a fixed order; the result is valid in thread 0.
// `scratch` holds >= 32 doubles; the call ends with a barrier so the scratch
// can be reused immediately.
template <class Op>
__device__ __forceinline__ double block_reduce(double v, double* scratch, Op op) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = (lane < nw) ? scratch[lane] : Op::identity;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    __syncthreads();
    return v;
}

// Deterministic reduction of `count` block partials by one block.
template <class Op>
__device__ __forceinline__ double reduce_partials(const double* p, int count, double* scratch, Op op) {
    double v = Op::identity;
    for (int i = threadIdx.x; i < count; i += blockDim.x) v = op(v, p[i]);
    return block_reduce(v, scratch, op);
}

}  // namespace mc
