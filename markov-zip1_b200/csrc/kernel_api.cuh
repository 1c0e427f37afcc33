// Kernel-level entry points of the C ABI (device pointers, the context's
// stream): SpMV, the device transpose and Ruiz equilibration on their own.
// Included once, by engine.cu.
#pragma once

#include "engine.hpp"
#include "solve.cuh"

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

}  // extern "C"
