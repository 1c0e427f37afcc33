// equilibrate() of markov-cero on the B200 engine; see ruiz_gpu.hpp.  The
// canonical CSC's size_t offsets and indices become int32 device arrays; the
// values, rhs and objective go to the device, are scaled there and come back.
#include "ruiz_gpu.hpp"

#include "mc_pdlp.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace markov_cero::scale {

namespace {

[[noreturn]] void fail(int code, const char* what) {
    char msg[512];
    mc_last_error(msg, sizeof msg);
    const std::string text = std::string(what) + ": " + msg;
    if (code == MC_ERR_INVALID_ARGUMENT) throw std::invalid_argument(text);
    if (code == MC_ERR_RESOURCE_LIMIT) throw std::length_error(text);
    throw std::runtime_error(text);
}

int32_t to_int32(std::size_t v) {
    if (v > static_cast<std::size_t>(std::numeric_limits<int32_t>::max()))
        throw std::length_error("GPU equilibrate: index beyond the engine's int32 range");
    return static_cast<int32_t>(v);
}

struct ThreadContext {
    mc_pdlp_ctx* ctx = nullptr;
    ~ThreadContext() {
        if (ctx) mc_pdlp_ctx_destroy(ctx);
    }
    mc_pdlp_ctx* get() {
        if (!ctx) {
            const int rc = mc_pdlp_ctx_create(0, &ctx);
            if (rc != MC_OK) {
                ctx = nullptr;
                fail(rc, "GPU equilibrate (no CPU fallback)");
            }
        }
        return ctx;
    }
};
thread_local ThreadContext g_ctx;

// device buffers of one call, freed on every path
struct Device {
    std::vector<void*> ptrs;
    ~Device() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    T* alloc(std::size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, (count ? count : 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("GPU equilibrate: device allocation failed");
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

void copy(void* dst, const void* src, std::size_t bytes, cudaMemcpyKind kind) {
    if (bytes && cudaMemcpy(dst, src, bytes, kind) != cudaSuccess) {
        cudaGetLastError();
        throw std::runtime_error("GPU equilibrate: copy failed");
    }
}

}  // namespace

RuizScalers equilibrate_gpu(transform::SparseCanonicalModel& model, const RuizOptions& options) {
    const auto& A = model.matrix;
    const std::size_t m = A.rows, n = A.columns, nnz = A.values.size();
    RuizScalers out;
    out.row_scale.assign(m, 1.0);
    out.col_scale.assign(n, 1.0);
    out.inv_row_scale.assign(m, 1.0);
    out.inv_col_scale.assign(n, 1.0);
    if (m == 0 || n == 0 || nnz == 0) return out;  // ruiz_scaling.cpp:30-32
    if (A.column_offsets.size() != n + 1 || A.row_indices.size() != nnz || model.rhs.size() != m ||
        model.objective.size() != n)
        throw std::invalid_argument("GPU equilibrate: model arrays do not match the matrix dimensions");
    std::vector<int32_t> cs(n + 1), ri(nnz);
    for (std::size_t j = 0; j <= n; ++j) cs[j] = to_int32(A.column_offsets[j]);
    for (std::size_t p = 0; p < nnz; ++p) ri[p] = to_int32(A.row_indices[p]);
    mc_pdlp_ctx* ctx = g_ctx.get();
    Device d;
    int32_t* dcs = d.alloc<int32_t>(n + 1);
    int32_t* dri = d.alloc<int32_t>(nnz);
    double* dv = d.alloc<double>(nnz);
    double* drhs = d.alloc<double>(m);
    double* dobj = d.alloc<double>(n);
    double* drs = d.alloc<double>(m);
    double* dcsc = d.alloc<double>(n);
    double* dirs = d.alloc<double>(m);
    double* dics = d.alloc<double>(n);
    copy(dcs, cs.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice);
    copy(dri, ri.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice);
    copy(dv, A.values.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice);
    copy(drhs, model.rhs.data(), sizeof(double) * m, cudaMemcpyHostToDevice);
    copy(dobj, model.objective.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
    int64_t iterations = 0;
    int32_t converged = 0;
    const int rc = mc_ruiz_equilibrate_canonical(ctx, to_int32(m), to_int32(n), static_cast<int64_t>(nnz), dcs, dri,
                                                 dv, drhs, dobj, static_cast<int64_t>(options.max_iterations),
                                                 options.tolerance, options.min_scale, options.max_scale, drs, dcsc,
                                                 dirs, dics, &iterations, &converged);
    if (rc != MC_OK) fail(rc, "GPU equilibrate");
    copy(model.matrix.values.data(), dv, sizeof(double) * nnz, cudaMemcpyDeviceToHost);
    copy(model.rhs.data(), drhs, sizeof(double) * m, cudaMemcpyDeviceToHost);
    copy(model.objective.data(), dobj, sizeof(double) * n, cudaMemcpyDeviceToHost);
    copy(out.row_scale.data(), drs, sizeof(double) * m, cudaMemcpyDeviceToHost);
    copy(out.col_scale.data(), dcsc, sizeof(double) * n, cudaMemcpyDeviceToHost);
    copy(out.inv_row_scale.data(), dirs, sizeof(double) * m, cudaMemcpyDeviceToHost);
    copy(out.inv_col_scale.data(), dics, sizeof(double) * n, cudaMemcpyDeviceToHost);
    out.iterations_executed = static_cast<std::size_t>(iterations);
    out.converged = converged != 0;
    return out;
}

}  // namespace markov_cero::scale
