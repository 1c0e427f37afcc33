// Host driver of the B200 PDLP engine and the C ABI of include/mc_pdlp.h.
//
// A solve (the GPU form of solve_pdlp, src/lp/first_order/pdlp.cpp:139-276):
//   1. copy the model into the context's arena (one allocation, reused);
//   2. validate it on the device (every later gather stays in bounds);
//   3. build CSR(A) from CSC(A) on the device, rows in ascending column order;
//   4. Ruiz equilibration of both copies (ruiz_scaling.cpp:152-247);
//   5. norms, step sizes and the starting point;
//   6. the PDHG loop in chunks of restart_every iterations, each chunk one
//      CUDA graph replay (2 fused SpMV kernels per iteration plus the
//      step-size probe every 10th iteration, then the KKT residual pass and
//      the restart logic, all on the device); the host polls one flag per
//      chunk, one chunk behind, so the GPU never idles between chunks;
//   7. unscale the averages and copy them out.
#include "mc_pdlp.h"
#include "mc_pdlp_testing.h"

#include "engine.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace mc {

// ------------------------------------------------------------------ errors
static thread_local std::string g_error;
static int g_inject_alloc_failures = 0;

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what, int line) {
    const int code = (e == cudaErrorMemoryAllocation) ? MC_ERR_OUT_OF_MEMORY
                     : (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice ||
                        e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
                         ? MC_ERR_NO_DEVICE
                         : MC_ERR_CUDA;
    return set_error(code, "%s failed at engine.cu:%d: %s", what, line, cudaGetErrorString(e));
}

int check_device(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return set_error(MC_ERR_NO_DEVICE, "no CUDA device (%s); the engine has no CPU fallback",
                         e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return set_error(MC_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, count);
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(MC_ERR_NO_DEVICE, "device %d is sm_%d%d; this engine is built for sm_100a",
                         device, prop.major, prop.minor);
    return MC_OK;
}

// ----------------------------------------------------------------- arena
int Arena::reserve(size_t bytes) {
    if (bytes <= capacity) return MC_OK;
    if (base) {
        cudaFree(base);
        base = nullptr;
        capacity = 0;
    }
    if (g_inject_alloc_failures > 0) {
        --g_inject_alloc_failures;
        return set_error(MC_ERR_OUT_OF_MEMORY, "injected allocation failure (%zu bytes)", bytes);
    }
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) {
        base = nullptr;
        cudaGetLastError();
        return cuda_fail(e, "cudaMalloc(arena)", __LINE__);
    }
    capacity = bytes;
    return MC_OK;
}

// ------------------------------------------------------------------ context
Ctx::~Ctx() {
    if (device >= 0) cudaSetDevice(device);
    drop_session();
    release_graphs();
    if (arena.base) cudaFree(arena.base);
    if (h_state) cudaFreeHost(h_state);
    for (auto& e : prof_events) cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_a, ev_b, ev_c, ev_d, ev_poll[0], ev_poll[1]})
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
}

void Ctx::release_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
}

int Ctx::init(int dev) {
    TRY(check_device(dev));
    device = dev;
    CU(cudaSetDevice(dev));
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CU(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    CU(cudaEventCreate(&ev_a));
    CU(cudaEventCreate(&ev_b));
    CU(cudaEventCreate(&ev_c));
    CU(cudaEventCreate(&ev_d));
    CU(cudaEventCreateWithFlags(&ev_poll[0], cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&ev_poll[1], cudaEventDisableTiming));
    CU(cudaMallocHost(reinterpret_cast<void**>(&h_state), sizeof(DevState) * 4));
    return MC_OK;
}

// ------------------------------------------------------- launch bookkeeping
void Ctx::begin_launch(int kind) {
    launches[kind] += 1;
    if (profiling && !capturing) {
        if (prof_used + 2 > prof_events.size()) {
            for (int q = 0; q < 64; ++q) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                prof_events.push_back(e);
            }
        }
        cudaEventRecord(prof_events[prof_used], stream);
        pending.push_back({kind, (int)prof_used});
        prof_used += 2;
    }
}

void Ctx::end_launch() {
    if (profiling && !capturing) cudaEventRecord(prof_events[pending.back().first_event + 1], stream);
}

int Ctx::drain_profile() {
    if (!profiling || pending.empty()) return MC_OK;
    CU(cudaStreamSynchronize(stream));
    for (const auto& p : pending) {
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, prof_events[p.first_event], prof_events[p.first_event + 1]));
        kernel_ms[p.kind] += ms;
    }
    pending.clear();
    prof_used = 0;
    return MC_OK;
}

int Ctx::launch_check(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what, __LINE__);
    return MC_OK;
}

int blocks_for(const Ctx& ctx, long long work_items, int per_block) {
    long long b = (work_items + per_block - 1) / per_block;
    const long long cap = std::min<long long>((long long)ctx.sm_count * (2048 / kBlock), kMaxPartials / 2);
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Lanes per line for the lane kernels: each lane should carry about four
// entries (four loads in flight per step), up to a warp per line.
int pick_lanes(double mean_len) {
    int g = 1;
    while (g < 32 && 4.0 * (2 * g) <= mean_len) g *= 2;
    return g;
}

}  // namespace mc

#include "solve.cuh"
#include "batch.cuh"
#include "variants.cuh"
#include "kernel_api.cuh"
#include "verify.cuh"
#include "presolve.cuh"

namespace mc {
// The learned warm start's large instances use the engine's device transpose
// (rows in ascending column order): an auxiliary context and the CSR of a
// device CSC.  Declared in gnn.cu.
Ctx* aux_ctx_create(int device) {
    Ctx* c = new Ctx();
    if (c->init(device) != MC_OK) {
        delete c;
        return nullptr;
    }
    return c;
}

void aux_ctx_destroy(Ctx* c) { delete c; }

int aux_csr(Ctx* c, int m, int n, long long nnz, const int* cs, const int* ri, const double* v, int* rs, int* ci,
            double* rv) {
    cudaStream_t s = c->stream;
    int *cursor = nullptr, *long_rows = nullptr, *counters = nullptr, *scan = nullptr;
    const size_t scan_ints = (size_t)(m + 1) / kScanTile + 4096;
    int rc = MC_OK;
    auto get = [&](int** p, size_t count) {
        if (rc == MC_OK && cudaMallocAsync(reinterpret_cast<void**>(p), sizeof(int) * count, s) != cudaSuccess)
            rc = set_error(MC_ERR_OUT_OF_MEMORY, "transpose scratch");
    };
    get(&cursor, (size_t)m + 1);
    get(&long_rows, (size_t)m + 1);
    get(&counters, 4);
    get(&scan, scan_ints);
    if (rc == MC_OK) rc = build_csr(*c, m, n, nnz, cs, ri, v, rs, ci, rv, cursor, long_rows, counters, scan);
    for (int* p : {cursor, long_rows, counters, scan})
        if (p) cudaFreeAsync(p, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && rc == MC_OK) rc = set_error(MC_ERR_CUDA, "transpose");
    return rc;
}
}  // namespace mc

using namespace mc;

// =================================================================== C ABI
extern "C" {

int mc_pdlp_abi_version(void) { return MC_PDLP_ABI_VERSION; }

void mc_pdlp_default_options(mc_pdlp_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->max_iterations = 100000;
    o->restart_every = 40;
    o->primal_tolerance = 1e-4;
    o->dual_tolerance = 1e-4;
    o->gap_tolerance = 1e-4;
    o->step_size_reduction = 0.9;
    o->power_iterations = 20;
    o->backend = MC_BACKEND_GPU;
    o->restart_strategy = MC_RESTART_ADAPTIVE;
    o->restart_reduction_factor = 0.368;
    o->adaptive_step_size = 1;
    o->adaptive_primal_weight = 1;
    o->initial_primal_weight = 0.0;
    o->primal_weight_smoothing = 0.5;
    o->ruiz_scaling = 1;
    o->ruiz_iterations = 10;
    o->precision = MC_PRECISION_FP64;
    o->device = 0;
    o->profile_kernels = 0;
    o->check_every_chunks = 1;
}

int mc_pdlp_struct_sizes(size_t* sizes, int count) {
    const size_t all[8] = {sizeof(mc_lp),           sizeof(mc_pdlp_options),    sizeof(mc_pdlp_result),
                           sizeof(mc_pdlp_trace),   sizeof(mc_verify_report),   sizeof(mc_canonical_lp),
                           sizeof(mc_presolve_options), sizeof(mc_presolve_info)};
    if (!sizes || count < 0) return set_error(MC_ERR_INVALID_ARGUMENT, "bad sizes buffer");
    for (int q = 0; q < count && q < 8; ++q) sizes[q] = all[q];
    return MC_OK;
}

int mc_last_error(char* buffer, size_t length) {
    if (buffer && length) std::snprintf(buffer, length, "%s", g_error.c_str());
    return MC_OK;
}

int mc_device_count(int* count) {
    if (!count) return set_error(MC_ERR_INVALID_ARGUMENT, "count is NULL");
    *count = 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return MC_OK;
    }
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10) ++*count;
    }
    return MC_OK;
}

int mc_pdlp_ctx_create(int device, mc_pdlp_ctx** out) {
    if (!out) return set_error(MC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    auto* ctx = new (std::nothrow) Ctx();
    if (!ctx) return set_error(MC_ERR_OUT_OF_MEMORY, "host allocation failed");
    DeviceGuard guard(device);
    const int rc = ctx->init(device);
    if (rc != MC_OK) {
        delete ctx;
        return rc;
    }
    *out = reinterpret_cast<mc_pdlp_ctx*>(ctx);
    return MC_OK;
}

int mc_pdlp_ctx_destroy(mc_pdlp_ctx* c) {
    delete reinterpret_cast<Ctx*>(c);
    return MC_OK;
}

int mc_pdlp_ctx_solve(mc_pdlp_ctx* c, const mc_lp* lp, const mc_pdlp_options* options,
                      const double* initial_primal, const double* initial_dual, double* primal_out,
                      double* dual_out, mc_pdlp_result* result, mc_pdlp_trace* trace) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return solve_lp(*ctx, lp, options, initial_primal, initial_dual, primal_out, dual_out, result,
                    trace);
}

int mc_pdlp_ctx_stream(mc_pdlp_ctx* c, void** stream) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx || !stream) return set_error(MC_ERR_INVALID_ARGUMENT, "context or stream is NULL");
    *stream = reinterpret_cast<void*>(ctx->stream);
    return MC_OK;
}

int mc_pdlp_ctx_begin(mc_pdlp_ctx* c, const mc_lp* lp, const mc_pdlp_options* options,
                      const double* initial_primal, const double* initial_dual, mc_pdlp_trace* trace) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    const int rc = begin_session(*ctx, lp, options, initial_primal, initial_dual, trace);
    if (rc != MC_OK) ctx->drop_session();
    return rc;
}

int mc_pdlp_ctx_iterate(mc_pdlp_ctx* c, int64_t chunks, int64_t* iterations, int32_t* finished) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    long long it = 0;
    int fin = 0;
    const int rc = iterate_session(*ctx, (long long)chunks, &it, &fin);
    if (rc != MC_OK) {
        ctx->drop_session();
        return rc;
    }
    if (iterations) *iterations = it;
    if (finished) *finished = fin;
    return MC_OK;
}

int mc_pdlp_ctx_finish(mc_pdlp_ctx* c, double* primal_out, double* dual_out, mc_pdlp_result* result) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    const int rc = finish_session(*ctx, primal_out, dual_out, result);
    if (rc != MC_OK) ctx->drop_session();
    return rc;
}

int mc_pdlp_ctx_solve_batch(mc_pdlp_ctx* c, const mc_lp* lps, int32_t count, const mc_pdlp_options* options,
                            double* const* primal_out, double* const* dual_out, mc_pdlp_result* results) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return solve_batch(*ctx, lps, count, options, nullptr, nullptr, primal_out, dual_out, results);
}

int mc_pdlp_ctx_solve_batch_warm(mc_pdlp_ctx* c, const mc_lp* lps, int32_t count, const mc_pdlp_options* options,
                                 const double* const* initial_primal, const double* const* initial_dual,
                                 double* const* primal_out, double* const* dual_out, mc_pdlp_result* results) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return solve_batch(*ctx, lps, count, options, initial_primal, initial_dual, primal_out, dual_out, results);
}

int mc_pdlp_ctx_solve_variants(mc_pdlp_ctx* c, const mc_lp* base, int32_t count, const double* const* var_lower,
                               const double* const* var_upper, const mc_pdlp_options* options,
                               const double* const* initial_primal, const double* const* initial_dual,
                               double* const* primal_out, double* const* dual_out, mc_pdlp_result* results) {
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return solve_variants(*ctx, base, count, var_lower, var_upper, options, initial_primal, initial_dual,
                          primal_out, dual_out, results);
}

int mc_pdlp_solve(const mc_lp* lp, const mc_pdlp_options* options, const double* initial_primal,
                  const double* initial_dual, double* primal_out, double* dual_out,
                  mc_pdlp_result* result) {
    TRY(validate_options(options));
    TRY(validate_lp(lp));
    mc_pdlp_ctx* c = nullptr;
    TRY(mc_pdlp_ctx_create(options->device, &c));
    const int rc = mc_pdlp_ctx_solve(c, lp, options, initial_primal, initial_dual, primal_out,
                                     dual_out, result, nullptr);
    mc_pdlp_ctx_destroy(c);
    return rc;
}

int mc_test_inject_alloc_failures(int count) {
    g_inject_alloc_failures = count;
    return MC_OK;
}

}  // extern "C"
