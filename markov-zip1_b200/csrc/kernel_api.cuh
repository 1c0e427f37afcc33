// Kernel-level entry points of the C ABI (device pointers, the context's
// stream): SpMV, the device transpose and Ruiz equilibration on their own.
// Included once, by engine.cu.
#pragma once

#include "engine.hpp"
#include "solve.cuh"

#include <cmath>

namespace mc {

// Ruiz bound/objective scaling of a model (ruiz_scaling.cpp:221-244), in place.
__global__ void k_ruiz_apply(int m, int n, const double* __restrict__ row_scale,
                             const double* __restrict__ col_scale, double* __restrict__ objective,
                             double* __restrict__ var_lower, double* __restrict__ var_upper,
                             double* __restrict__ row_lower, double* __restrict__ row_upper) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
        if (t < n) {
            const double s = col_scale[t];
            const double inv = 1.0 / s;
            if (isfinite(var_lower[t])) var_lower[t] = __dmul_rn(var_lower[t], inv);
            if (isfinite(var_upper[t])) var_upper[t] = __dmul_rn(var_upper[t], inv);
            objective[t] = __dmul_rn(objective[t], s);
        } else {
            const int i = t - n;
            const double s = row_scale[i];
            if (isfinite(row_lower[i])) row_lower[i] = __dmul_rn(row_lower[i], s);
            if (isfinite(row_upper[i])) row_upper[i] = __dmul_rn(row_upper[i], s);
        }
    }
}

// The canonical path's finish (ruiz_scaling.cpp:106-122): scales clamped to
// [min_scale, max_scale], their inverses, rhs scaled by the clamped row scale
// and the objective by the clamped column scale; a non-finite result sets
// *bad (1 rhs, 2 objective).
__global__ void k_ruiz_canonical_finish(int m, int n, double min_scale, double max_scale,
                                        double* __restrict__ row_scale, double* __restrict__ col_scale,
                                        double* __restrict__ inv_row, double* __restrict__ inv_col,
                                        double* __restrict__ rhs, double* __restrict__ objective,
                                        int* __restrict__ bad) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m + n; t += gridDim.x * blockDim.x) {
        if (t < m) {
            const double s = clampv(row_scale[t], min_scale, max_scale);
            row_scale[t] = s;
            inv_row[t] = __ddiv_rn(1.0, s);
            const double r = __dmul_rn(rhs[t], s);
            rhs[t] = r;
            if (!isfinite(r)) atomicOr(bad, 1);
        } else {
            const int j = t - m;
            const double s = clampv(col_scale[j], min_scale, max_scale);
            col_scale[j] = s;
            inv_col[j] = __ddiv_rn(1.0, s);
            const double c = __dmul_rn(objective[j], s);
            objective[j] = c;
            if (!isfinite(c)) atomicOr(bad, 2);
        }
    }
}

}  // namespace mc

using namespace mc;

extern "C" {

int mc_spmv_csr(mc_pdlp_ctx* c, int32_t m, int32_t n, const int32_t* row_start, const int32_t* col_index,
                const double* value, const double* x, double* y) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || m < 0 || n < 0 || !row_start || !x || !y) return set_error(MC_ERR_INVALID_ARGUMENT, "bad spmv arguments");
    if (m == 0) return MC_OK;
    DeviceGuard guard(ctx->device);
    long long nnz = 0;
    int last = 0;
    CU(cudaMemcpy(&last, row_start + m, sizeof(int), cudaMemcpyDeviceToHost));
    nnz = last;
    const int g = pick_lanes((double)nnz / m);
    const int nb = blocks_for(*ctx, m, kBlock / g);
    MC_DISPATCH_G(g, (k_spmv<G, double><<<nb, kBlock, 0, ctx->stream>>>(m, row_start, col_index, value, x, y)));
    TRY(ctx->launch_check("mc_spmv_csr"));
    CU(cudaStreamSynchronize(ctx->stream));
    return MC_OK;
}

int mc_csc_to_csr(mc_pdlp_ctx* c, int32_t m, int32_t n, int64_t nnz, const int32_t* col_start,
                  const int32_t* row_index, const double* value, int32_t* row_start, int32_t* col_index,
                  double* csr_value) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || m < 0 || n < 0 || nnz < 0 || !col_start || !row_start)
        return set_error(MC_ERR_INVALID_ARGUMENT, "bad transpose arguments");
    DeviceGuard guard(ctx->device);
    cudaStream_t s = ctx->stream;
    int *cursor = nullptr, *long_rows = nullptr, *counters = nullptr, *scan = nullptr;
    const size_t scan_ints = (size_t)(m + 1) / kScanTile + 4096;
    CU(cudaMallocAsync(reinterpret_cast<void**>(&cursor), sizeof(int) * (size_t)(m + 1), s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&long_rows), sizeof(int) * (size_t)(m + 1), s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&counters), sizeof(int) * 4, s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&scan), sizeof(int) * scan_ints, s));
    if (n > 0 && nnz > 0) {
        int* bad = counters + 2;
        CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
        k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, col_start, row_index, value, bad);
        int hbad = 0;
        CU(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (hbad) {
            cudaFreeAsync(cursor, s);
            cudaFreeAsync(long_rows, s);
            cudaFreeAsync(counters, s);
            cudaFreeAsync(scan, s);
            return set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix (flags %d)", hbad);
        }
    }
    const int rc = build_csr(*ctx, m, n, nnz, col_start, row_index, value, row_start, col_index, csr_value,
                             cursor, long_rows, counters, scan);
    cudaFreeAsync(cursor, s);
    cudaFreeAsync(long_rows, s);
    cudaFreeAsync(counters, s);
    cudaFreeAsync(scan, s);
    TRY(rc);
    CU(cudaStreamSynchronize(s));
    return MC_OK;
}

int mc_ruiz_equilibrate(mc_pdlp_ctx* c, int32_t m, int32_t n, int64_t nnz, const int32_t* col_start,
                        const int32_t* row_index, double* csc_value, const int32_t* row_start,
                        const int32_t* col_index, double* csr_value, double* objective, double* var_lower,
                        double* var_upper, double* row_lower, double* row_upper, int64_t max_iterations,
                        double* row_scale, double* col_scale, int64_t* iterations_executed) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || m < 0 || n < 0 || nnz < 0 || max_iterations < 0 || !row_scale || !col_scale)
        return set_error(MC_ERR_INVALID_ARGUMENT, "bad Ruiz arguments");
    DeviceGuard guard(ctx->device);
    cudaStream_t s = ctx->stream;
    double *r_tmp = nullptr, *c_tmp = nullptr, *partials = nullptr;
    DevState* st = nullptr;
    CU(cudaMallocAsync(reinterpret_cast<void**>(&r_tmp), sizeof(double) * (size_t)(m + 1), s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&c_tmp), sizeof(double) * (size_t)(n + 1), s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&partials), sizeof(double) * NUM_SLOTS * kMaxPartials, s));
    CU(cudaMallocAsync(reinterpret_cast<void**>(&st), sizeof(DevState), s));
    CU(cudaMemsetAsync(st, 0, sizeof(DevState), s));
    int rc = MC_OK;
    if (m > 0 && n > 0) {
        rc = ruiz(*ctx, m, n, nnz, col_start, row_index, csc_value, row_start, col_index, csr_value, row_scale,
                  col_scale, r_tmp, c_tmp, partials, st, max_iterations);
        if (rc == MC_OK && objective && var_lower && var_upper && row_lower && row_upper) {
            k_ruiz_apply<<<blocks_for(*ctx, (long long)n + m, kBlock), kBlock, 0, s>>>(
                m, n, row_scale, col_scale, objective, var_lower, var_upper, row_lower, row_upper);
            rc = ctx->launch_check("k_ruiz_apply");
        }
    }
    DevState h;
    std::memset(&h, 0, sizeof h);
    const cudaError_t e = cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(r_tmp, s);
    cudaFreeAsync(c_tmp, s);
    cudaFreeAsync(partials, s);
    cudaFreeAsync(st, s);
    TRY(rc);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(state)", __LINE__);
    CU(cudaStreamSynchronize(s));
    if (iterations_executed) *iterations_executed = h.ruiz_passes;
    return MC_OK;
}

int mc_ruiz_equilibrate_canonical(mc_pdlp_ctx* c, int32_t m, int32_t n, int64_t nnz, const int32_t* col_start,
                                  const int32_t* row_index, double* value, double* rhs, double* objective,
                                  int64_t max_iterations, double tolerance, double min_scale, double max_scale,
                                  double* row_scale, double* col_scale, double* inv_row_scale,
                                  double* inv_col_scale, int64_t* iterations_executed, int32_t* converged) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || m < 0 || n < 0 || nnz < 0 || max_iterations < 0 || !row_scale || !col_scale || !inv_row_scale ||
        !inv_col_scale || (m > 0 && !rhs) || (n > 0 && !objective))
        return set_error(MC_ERR_INVALID_ARGUMENT, "bad canonical Ruiz arguments");
    if (!std::isfinite(tolerance) || tolerance < 0.0 || !std::isfinite(min_scale) || !std::isfinite(max_scale) ||
        !(min_scale > 0.0) || min_scale > max_scale)
        return set_error(MC_ERR_INVALID_ARGUMENT, "bad canonical Ruiz options");
    DeviceGuard guard(ctx->device);
    cudaStream_t s = ctx->stream;
    if (iterations_executed) *iterations_executed = 0;
    if (converged) *converged = 0;
    // every scale 1 first (also the answer for an empty model, returned
    // before the clamp as the reference does, ruiz_scaling.cpp:30-32)
    for (double* v : {row_scale, inv_row_scale})
        if (m > 0) {
            k_fill<double><<<blocks_for(*ctx, m, kBlock), kBlock, 0, s>>>(v, m, 1.0);
        }
    for (double* v : {col_scale, inv_col_scale})
        if (n > 0) {
            k_fill<double><<<blocks_for(*ctx, n, kBlock), kBlock, 0, s>>>(v, n, 1.0);
        }
    TRY(ctx->launch_check("canonical Ruiz fill"));
    if (m == 0 || n == 0 || nnz == 0) {
        CU(cudaStreamSynchronize(s));
        return MC_OK;
    }
    int *rs = nullptr, *ci = nullptr, *cursor = nullptr, *long_rows = nullptr, *counters = nullptr, *scan = nullptr;
    double *rv = nullptr, *r_tmp = nullptr, *c_tmp = nullptr, *partials = nullptr;
    DevState* st = nullptr;
    const size_t scan_ints = (size_t)(m + 1) / kScanTile + 4096;
    int rc = MC_OK;
    auto alloc = [&](void** p, size_t bytes) {
        if (rc == MC_OK && cudaMallocAsync(p, bytes, s) != cudaSuccess)
            rc = set_error(MC_ERR_OUT_OF_MEMORY, "canonical Ruiz scratch (%zu bytes)", bytes);
    };
    alloc(reinterpret_cast<void**>(&rs), sizeof(int) * (size_t)(m + 1));
    alloc(reinterpret_cast<void**>(&ci), sizeof(int) * (size_t)(nnz + 1));
    alloc(reinterpret_cast<void**>(&rv), sizeof(double) * (size_t)(nnz + 1));
    alloc(reinterpret_cast<void**>(&cursor), sizeof(int) * (size_t)(m + 1));
    alloc(reinterpret_cast<void**>(&long_rows), sizeof(int) * (size_t)(m + 1));
    alloc(reinterpret_cast<void**>(&counters), sizeof(int) * 4);
    alloc(reinterpret_cast<void**>(&scan), sizeof(int) * scan_ints);
    alloc(reinterpret_cast<void**>(&r_tmp), sizeof(double) * (size_t)(m + 1));
    alloc(reinterpret_cast<void**>(&c_tmp), sizeof(double) * (size_t)(n + 1));
    alloc(reinterpret_cast<void**>(&partials), sizeof(double) * NUM_SLOTS * kMaxPartials);
    alloc(reinterpret_cast<void**>(&st), sizeof(DevState));
    DevState h;
    std::memset(&h, 0, sizeof h);
    int hbad = 0;
    if (rc == MC_OK) {
        cudaMemsetAsync(counters, 0, sizeof(int) * 4, s);
        cudaMemsetAsync(st, 0, sizeof(DevState), s);
        k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, col_start, row_index, value,
                                                                   counters + 2);
        if (cudaMemcpyAsync(&hbad, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = set_error(MC_ERR_CUDA, "canonical Ruiz validation");
        else if (hbad)
            rc = set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix (flags %d)", hbad);
    }
    // the loop runs on the CSC and a CSR copy (row maxima), as ruiz() does for
    // the PDLP path; only the CSC values are the caller's
    if (rc == MC_OK) rc = build_csr(*ctx, m, n, nnz, col_start, row_index, value, rs, ci, rv, cursor, long_rows,
                                    counters, scan);
    if (rc == MC_OK) rc = ruiz(*ctx, m, n, nnz, col_start, row_index, value, rs, ci, rv, row_scale, col_scale, r_tmp,
                              c_tmp, partials, st, max_iterations, tolerance);
    if (rc == MC_OK) {
        cudaMemsetAsync(counters, 0, sizeof(int) * 4, s);
        k_ruiz_canonical_finish<<<blocks_for(*ctx, (long long)m + n, kBlock), kBlock, 0, s>>>(
            m, n, min_scale, max_scale, row_scale, col_scale, inv_row_scale, inv_col_scale, rhs, objective,
            counters);
        rc = ctx->launch_check("k_ruiz_canonical_finish");
    }
    if (rc == MC_OK && (cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                        cudaMemcpyAsync(&hbad, counters, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess))
        rc = set_error(MC_ERR_CUDA, "canonical Ruiz read-back");
    for (void* p : {(void*)rs, (void*)ci, (void*)rv, (void*)cursor, (void*)long_rows, (void*)counters, (void*)scan,
                    (void*)r_tmp, (void*)c_tmp, (void*)partials, (void*)st})
        if (p) cudaFreeAsync(p, s);
    TRY(rc);
    CU(cudaStreamSynchronize(s));
    // the reference throws overflow_error here (ruiz_scaling.cpp:112-121)
    if (hbad & 1) return set_error(MC_ERR_INVALID_ARGUMENT, "non-finite scaled RHS");
    if (hbad & 2) return set_error(MC_ERR_INVALID_ARGUMENT, "non-finite scaled objective");
    if (iterations_executed) *iterations_executed = h.ruiz_passes;
    if (converged) *converged = h.ruiz_done ? 1 : 0;
    return MC_OK;
}

}  // extern "C"
