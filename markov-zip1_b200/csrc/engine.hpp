// Host-side types of the engine (one translation unit: engine.cu).
#pragma once

#include "mc_pdlp.h"
#include "common.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <tuple>
#include <vector>

#define CU(call)                                                            \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) return ::mc::cuda_fail(e_, #call, __LINE__); \
    } while (0)

#define TRY(expr)                     \
    do {                              \
        const int rc_ = (expr);       \
        if (rc_ != MC_OK) return rc_; \
    } while (0)

namespace mc {

inline double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// RAII device switch for the calling thread.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int set_error(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, int line);
int check_device(int device);

// One device allocation carved into the arrays of a solve; grows, never shrinks.
struct Arena {
    void* base = nullptr;
    size_t capacity = 0;
    int reserve(size_t bytes);
};

// Bump allocator over a byte count, 256-byte aligned sub-arrays.
struct Layout {
    size_t offset = 0;
    template <class T>
    size_t add(long long count) {
        const size_t at = offset;
        offset += ((size_t)(count > 0 ? count : 1) * sizeof(T) + 255) & ~(size_t)255;
        return at;
    }
};

struct Session;                 // a stepwise solve in progress (solve.cuh)
void free_session(Session* s);

struct Ctx {
    int device = -1;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    Arena arena;
    DevState* h_state = nullptr;  // pinned, [4]
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_c = nullptr, ev_d = nullptr;
    cudaEvent_t ev_poll[2] = {nullptr, nullptr};
    std::map<int, cudaGraphExec_t> graphs;
    // batch lanes and tile size chosen by the autotuner, per batch shape (n, m, LPs, tiles):
    // lanes per column, lanes per row, block-steps per tile
    std::map<std::tuple<long long, long long, long long, long long, long long>, std::tuple<int, int, int>>
        lane_cache;

    // launch accounting / profiling
    bool profiling = false;
    bool capturing = false;
    long long launches[MC_KERNEL_KINDS] = {};
    double kernel_ms[MC_KERNEL_KINDS] = {};
    struct Pending {
        int kind;
        int first_event;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> prof_events;
    size_t prof_used = 0;

    // the stepwise solve in progress; any other use of the arena ends it
    Session* session = nullptr;

    ~Ctx();
    int init(int device);
    void drop_session() {
        free_session(session);
        session = nullptr;
    }
    void release_graphs();
    void begin_launch(int kind);
    void end_launch();
    int drain_profile();
    int launch_check(const char* what);
};

int blocks_for(const Ctx& ctx, long long work_items, int per_block);

// Grid for a grid-stride kernel: one full wave of resident blocks (from the
// kernel's own occupancy), never more than the work needs.
template <class K>
int grid_for(const Ctx& ctx, K kernel, long long work_items, int per_block, size_t smem = 0) {
    static thread_local std::map<const void*, int> cache;
    const void* key = reinterpret_cast<const void*>(kernel);
    auto it = cache.find(key);
    int per_sm = 0;
    if (it == cache.end()) {
        if (smem > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, smem) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        cache[key] = per_sm;
    } else {
        per_sm = it->second;
    }
    long long b = (work_items + per_block - 1) / per_block;
    const long long cap = std::min<long long>((long long)ctx.sm_count * per_sm, kMaxPartials / 2);
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}
int pick_lanes(double mean_len);

int solve_lp(Ctx& ctx, const mc_lp* lp, const mc_pdlp_options* o, const double* warm_x,
             const double* warm_y, double* x_out, double* y_out, mc_pdlp_result* res,
             mc_pdlp_trace* trace);
int begin_session(Ctx& ctx, const mc_lp* lp, const mc_pdlp_options* o, const double* warm_x,
                  const double* warm_y, mc_pdlp_trace* trace);
int iterate_session(Ctx& ctx, long long chunks, long long* iterations, int* finished);
int finish_session(Ctx& ctx, double* x_out, double* y_out, mc_pdlp_result* res);

}  // namespace mc
