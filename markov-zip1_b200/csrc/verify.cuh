// Post-solve verification of a primal candidate on the device
// (verify_primal, src/verify/primal_verifier.cpp:44-103).  Included once, by
// engine.cu after solve.cuh.
//
// The reference recomputes the row activities (SparseMatrixCSC::multiply,
// src/model/model.cpp:68-86) and the objective (primal_verifier.cpp:91-94)
// in long double on the host.  Here each row is summed by one thread in the
// reference's order (ascending column: CSR built on the device from the CSC)
// and, like the objective, in double-double arithmetic: products split
// exactly with an FMA (TwoProd), sums with Knuth's TwoSum, so the rounded
// result is at least as accurate as the long double one.  Block partials are
// reduced on the host in block order: the report is run-to-run identical.
#pragma once

#include "engine.hpp"
#include "solve.cuh"

#include <vector>

namespace mc {

struct DD {
    double hi, lo;
};

__host__ __device__ __forceinline__ DD dd_quick_sum(double a, double b) {  // |a| >= |b|
    const double s = a + b;
    return {s, b - (s - a)};
}

__host__ __device__ __forceinline__ DD dd_two_sum(double a, double b) {  // Knuth
    const double s = a + b;
    const double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}

__host__ __device__ __forceinline__ DD dd_add(DD a, DD b) {
    const DD s = dd_two_sum(a.hi, b.hi);
    return dd_quick_sum(s.hi, s.lo + (a.lo + b.lo));
}

// acc + a * b with the product split exactly by an FMA
__device__ __forceinline__ DD dd_add_product(DD acc, double a, double b) {
    const double p = __dmul_rn(a, b);
    const double e = __fma_rn(a, b, -p);
    return dd_add(acc, DD{p, e});
}

// Tolerance allowance, primal_verifier.cpp:9-15 (non-finite flagged by caller)
__host__ __device__ __forceinline__ double allowance(double actual, double expected, double abs_tol, double rel_tol) {
    const double big = fmax(1.0, fmax(fabs(actual), fabs(expected)));
    return abs_tol + rel_tol * big;
}

// Per-block results; field order fixed for the host reduction.
struct VerifyPart {
    DD objective;
    double max_var, max_row;
    long long count[4];
    long long first[4];
    int flags;  // 1 non-finite candidate, 2 allowance overflow, 4 non-finite activity
    int pad;
};

constexpr int kVerifyMaxBlocks = 2048;

__device__ __forceinline__ void note_violation(long long idx, int kind, long long* count, long long* first) {
    count[kind] += 1;
    if (first[kind] < 0 || idx < first[kind]) first[kind] = idx;
}

// one bound check (check_lower / check_upper, primal_verifier.cpp:16-37)
__device__ __forceinline__ void check_bound(double actual, double bound, bool lower, double abs_tol,
                                            double rel_tol, long long idx, int kind, double& maximum,
                                            long long* count, long long* first, int& flags) {
    if (!isfinite(bound)) return;
    const double magnitude = lower ? fmax(0.0, bound - actual) : fmax(0.0, actual - bound);
    const double permitted = allowance(actual, bound, abs_tol, rel_tol);
    if (!isfinite(permitted)) flags |= 2;
    maximum = fmax(maximum, magnitude);
    if (magnitude > permitted) note_violation(idx, kind, count, first);
}

// Block reduction of a VerifyPart into thread 0's copy (fixed order).
__device__ void reduce_part(VerifyPart& v, VerifyPart* shared) {
    shared[threadIdx.x] = v;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride) {
            VerifyPart& a = shared[threadIdx.x];
            const VerifyPart& b = shared[threadIdx.x + stride];
            a.objective = dd_add(a.objective, b.objective);
            a.max_var = fmax(a.max_var, b.max_var);
            a.max_row = fmax(a.max_row, b.max_row);
            for (int k = 0; k < 4; ++k) {
                a.count[k] += b.count[k];
                if (b.first[k] >= 0 && (a.first[k] < 0 || b.first[k] < a.first[k])) a.first[k] = b.first[k];
            }
            a.flags |= b.flags;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ VerifyPart empty_part() {
    VerifyPart v;
    v.objective = DD{0.0, 0.0};
    v.max_var = v.max_row = 0.0;
    for (int k = 0; k < 4; ++k) {
        v.count[k] = 0;
        v.first[k] = -1;
    }
    v.flags = 0;
    v.pad = 0;
    return v;
}

constexpr int kVerifyThreads = 128;

// variables: bounds (primal_verifier.cpp:60-68) and the objective terms
__global__ void __launch_bounds__(kVerifyThreads) k_verify_cols(int n, const double* __restrict__ x,
                                                                const double* __restrict__ lo,
                                                                const double* __restrict__ hi,
                                                                const double* __restrict__ obj, double abs_tol,
                                                                double rel_tol, VerifyPart* __restrict__ parts) {
    __shared__ VerifyPart sh[kVerifyThreads];
    VerifyPart v = empty_part();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double xj = x[j];
        if (!isfinite(xj)) {
            v.flags |= 1;
            continue;
        }
        check_bound(xj, lo[j], true, abs_tol, rel_tol, j, MC_VIOLATION_VARIABLE_LOWER, v.max_var, v.count, v.first,
                    v.flags);
        check_bound(xj, hi[j], false, abs_tol, rel_tol, j, MC_VIOLATION_VARIABLE_UPPER, v.max_var, v.count,
                    v.first, v.flags);
        v.objective = dd_add_product(v.objective, obj[j], xj);
    }
    reduce_part(v, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

// rows: activity in ascending column order, then the row bounds
// (primal_verifier.cpp:82-88)
__global__ void __launch_bounds__(kVerifyThreads) k_verify_rows(int m, const int* __restrict__ row_start,
                                                                const int* __restrict__ col_index,
                                                                const double* __restrict__ value,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ rlo,
                                                                const double* __restrict__ rhi, double abs_tol,
                                                                double rel_tol, VerifyPart* __restrict__ parts) {
    __shared__ VerifyPart sh[kVerifyThreads];
    VerifyPart v = empty_part();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        DD acc{0.0, 0.0};
        for (int p = row_start[i]; p < row_start[i + 1]; ++p) acc = dd_add_product(acc, value[p], x[col_index[p]]);
        const double activity = acc.hi + acc.lo;
        if (!isfinite(activity)) {
            v.flags |= 4;
            continue;
        }
        check_bound(activity, rlo[i], true, abs_tol, rel_tol, i, MC_VIOLATION_ROW_LOWER, v.max_row, v.count,
                    v.first, v.flags);
        check_bound(activity, rhi[i], false, abs_tol, rel_tol, i, MC_VIOLATION_ROW_UPPER, v.max_row, v.count,
                    v.first, v.flags);
    }
    reduce_part(v, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

static bool tolerance_ok(double v) { return std::isfinite(v) && v >= 0.0 && v <= 1e-4; }

int verify_primal(Ctx& ctx, const mc_lp* lp, const double* primal, double claimed, double feas_abs,
                  double feas_rel, double obj_abs, double obj_rel, mc_verify_report* rep) {
    ctx.drop_session();  // the verifier reuses the arena
    TRY(validate_lp(lp));
    if (!primal && lp->num_cols > 0) return set_error(MC_ERR_INVALID_ARGUMENT, "primal is NULL");
    // Tolerance::validate (primal_verifier.cpp:38-42)
    if (!tolerance_ok(feas_abs) || !tolerance_ok(feas_rel) || !tolerance_ok(obj_abs) || !tolerance_ok(obj_rel))
        return set_error(MC_ERR_INVALID_ARGUMENT, "tolerances must be finite and nonnegative");
    if (!std::isfinite(claimed)) return set_error(MC_ERR_INVALID_ARGUMENT, "claimed objective must be finite");
    const int m = lp->num_rows, n = lp->num_cols;
    const long long nnz = lp->nnz;
    const bool dev_in = lp->memory == MC_MEMORY_DEVICE;
    cudaStream_t s = ctx.stream;
    const int grid_c = std::max(1, std::min(kVerifyMaxBlocks, (n + kVerifyThreads - 1) / kVerifyThreads));
    const int grid_r = std::max(1, std::min(kVerifyMaxBlocks, (m + kVerifyThreads - 1) / kVerifyThreads));

    Layout L;
    const size_t o_cs = dev_in ? 0 : L.add<int>(n + 1);
    const size_t o_ri = dev_in ? 0 : L.add<int>(nnz + 1);
    const size_t o_cv = dev_in ? 0 : L.add<double>(nnz + 1);
    const size_t o_x = dev_in ? 0 : L.add<double>(n);
    const size_t o_obj = dev_in ? 0 : L.add<double>(n);
    const size_t o_lo = dev_in ? 0 : L.add<double>(n);
    const size_t o_hi = dev_in ? 0 : L.add<double>(n);
    const size_t o_rlo = dev_in ? 0 : L.add<double>(m);
    const size_t o_rhi = dev_in ? 0 : L.add<double>(m);
    const size_t o_rs = L.add<int>(m + 1);
    const size_t o_ci = L.add<int>(nnz + 1);
    const size_t o_rv = L.add<double>(nnz + 1);
    const size_t o_cursor = L.add<int>(m + 1);
    const size_t o_long = L.add<int>(m + 1);
    const size_t o_counters = L.add<int>(4);
    const size_t o_scan = L.add<int>((m + 1) / kScanTile + 4096);
    const size_t o_parts = L.add<VerifyPart>(2 * kVerifyMaxBlocks);
    TRY(ctx.arena.reserve(L.offset));
    char* A = static_cast<char*>(ctx.arena.base);
    auto at = [&](size_t off) { return static_cast<void*>(A + off); };
    auto input = [&](const void* src, size_t off, size_t bytes) -> const void* {
        if (dev_in) return src;
        if (bytes) {
            const cudaError_t e = cudaMemcpyAsync(at(off), src, bytes, cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return nullptr;
        }
        return at(off);
    };
    const int* cs = static_cast<const int*>(input(lp->col_start, o_cs, sizeof(int) * (size_t)(n + 1)));
    const int* ri = static_cast<const int*>(input(lp->row_index, o_ri, sizeof(int) * (size_t)nnz));
    const double* cv = static_cast<const double*>(input(lp->value, o_cv, sizeof(double) * (size_t)nnz));
    const double* x = static_cast<const double*>(input(primal, o_x, sizeof(double) * (size_t)n));
    const double* obj = static_cast<const double*>(input(lp->objective, o_obj, sizeof(double) * (size_t)n));
    const double* lo = static_cast<const double*>(input(lp->var_lower, o_lo, sizeof(double) * (size_t)n));
    const double* hi = static_cast<const double*>(input(lp->var_upper, o_hi, sizeof(double) * (size_t)n));
    const double* rlo = static_cast<const double*>(input(lp->row_lower, o_rlo, sizeof(double) * (size_t)m));
    const double* rhi = static_cast<const double*>(input(lp->row_upper, o_rhi, sizeof(double) * (size_t)m));
    if (!cs || !ri || !cv || !x || !obj || !lo || !hi || !rlo || !rhi)
        return cuda_fail(cudaGetLastError(), "cudaMemcpyAsync(verify inputs)", __LINE__);
    int* counters = static_cast<int*>(at(o_counters));
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    if (n > 0 && nnz > 0) {
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, cs, ri, cv, counters + 2);
        ctx.end_launch();
        int bad = 0;
        CU(cudaMemcpyAsync(&bad, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (bad) return set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix (flags %d)", bad);
    }
    int* rs = static_cast<int*>(at(o_rs));
    int* ci = static_cast<int*>(at(o_ci));
    double* rv = static_cast<double*>(at(o_rv));
    TRY(build_csr(ctx, m, n, nnz, cs, ri, cv, rs, ci, rv, static_cast<int*>(at(o_cursor)),
                  static_cast<int*>(at(o_long)), counters, static_cast<int*>(at(o_scan))));
    VerifyPart* parts = static_cast<VerifyPart*>(at(o_parts));
    ctx.begin_launch(MC_KERNEL_OTHER);
    k_verify_cols<<<grid_c, kVerifyThreads, 0, s>>>(n, x, lo, hi, obj, feas_abs, feas_rel, parts);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_OTHER);
    k_verify_rows<<<grid_r, kVerifyThreads, 0, s>>>(m, rs, ci, rv, x, rlo, rhi, feas_abs, feas_rel,
                                                     parts + kVerifyMaxBlocks);
    ctx.end_launch();
    TRY(ctx.launch_check("verify"));
    std::vector<VerifyPart> h(2 * kVerifyMaxBlocks);
    CU(cudaMemcpyAsync(h.data(), parts, sizeof(VerifyPart) * (size_t)grid_c, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(h.data() + kVerifyMaxBlocks, parts + kVerifyMaxBlocks, sizeof(VerifyPart) * (size_t)grid_r,
                       cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());

    // host reduction in block order
    DD objective{lp->objective_offset, 0.0};
    double max_var = 0.0, max_row = 0.0;
    long long count[4] = {0, 0, 0, 0}, first[4] = {-1, -1, -1, -1};
    int flags = 0;
    auto fold = [&](const VerifyPart& p) {
        objective = dd_add(objective, p.objective);
        max_var = std::max(max_var, p.max_var);
        max_row = std::max(max_row, p.max_row);
        for (int k = 0; k < 4; ++k) {
            count[k] += p.count[k];
            if (p.first[k] >= 0 && (first[k] < 0 || p.first[k] < first[k])) first[k] = p.first[k];
        }
        flags |= p.flags;
    };
    for (int b = 0; b < grid_c; ++b) fold(h[b]);
    for (int b = 0; b < grid_r; ++b) fold(h[kVerifyMaxBlocks + b]);
    if (flags & 1) return set_error(MC_ERR_INVALID_ARGUMENT, "candidate contains non-finite value");
    if (flags & 2) return set_error(MC_ERR_INVALID_ARGUMENT, "tolerance allowance overflow");
    if (flags & 4) return set_error(MC_ERR_INVALID_ARGUMENT, "matrix/vector product is non-finite");
    const double recomputed = objective.hi + objective.lo;
    if (!std::isfinite(recomputed)) return set_error(MC_ERR_INVALID_ARGUMENT, "recomputed objective is non-finite");

    std::memset(rep, 0, sizeof *rep);
    rep->recomputed_objective = recomputed;
    rep->objective_difference = std::fabs(recomputed - claimed);
    rep->maximum_row_violation = max_row;
    rep->maximum_variable_violation = max_var;
    for (int k = 0; k < 4; ++k) {
        rep->violations[k] = count[k];
        rep->first_index[k] = first[k];
    }
    const double obj_allow = allowance(recomputed, claimed, obj_abs, obj_rel);
    if (!std::isfinite(obj_allow)) return set_error(MC_ERR_INVALID_ARGUMENT, "tolerance allowance overflow");
    const bool obj_bad = rep->objective_difference > obj_allow;
    rep->violations[MC_VIOLATION_OBJECTIVE] = obj_bad ? 1 : 0;
    rep->first_index[MC_VIOLATION_OBJECTIVE] = obj_bad ? 0 : -1;
    long long total = 0;
    for (int k = 0; k < MC_VIOLATION_KINDS; ++k) total += rep->violations[k];
    rep->passed = total == 0 ? 1 : 0;
    return MC_OK;
}

}  // namespace mc

extern "C" int mc_verify_primal(mc_pdlp_ctx* c, const mc_lp* lp, const double* primal, double claimed_objective,
                                double feasibility_absolute, double feasibility_relative, double objective_absolute,
                                double objective_relative, mc_verify_report* report) {
    using namespace mc;
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || !lp || !report) return set_error(MC_ERR_INVALID_ARGUMENT, "bad verify arguments");
    DeviceGuard guard(ctx->device);
    return verify_primal(*ctx, lp, primal, claimed_objective, feasibility_absolute, feasibility_relative,
                         objective_absolute, objective_relative, report);
}
