// The FP64 solve driver (included once, by engine.cu).
#pragma once

#include "engine.hpp"
#include "iter_kernels.cuh"
#include "setup_kernels.cuh"
#include "mixed.cuh"

#include <climits>
#include <cmath>
#include <cstring>
#include <new>

namespace mc {

#define MC_DISPATCH_G(g, ...)                        \
    switch (g) {                                     \
        case 1: { constexpr int G = 1; __VA_ARGS__; } break;   \
        case 2: { constexpr int G = 2; __VA_ARGS__; } break;   \
        case 4: { constexpr int G = 4; __VA_ARGS__; } break;   \
        case 8: { constexpr int G = 8; __VA_ARGS__; } break;   \
        case 16: { constexpr int G = 16; __VA_ARGS__; } break; \
        default: { constexpr int G = 32; __VA_ARGS__; } break; \
    }

// Launch geometry of one problem: G lanes per line for each side, and grid
// sizes (one wave of resident blocks per kernel; the reduction partial counts
// follow the grids, so they are fixed per plan).
//
// (Tile-staged kernels -- one thread per line, the matrix slice of an
// nnz-balanced tile copied into shared memory with double-buffered cp.async --
// were built and measured on B200 at the 40M-nonzero LP: 0.406 / 0.307 ms
// per primal / dual launch against 0.244 / 0.245 for the lane kernels, so
// they were dropped.)
struct Plan {
    int g_col = 1, g_row = 1;
    int g_probe = 1;                      // lanes per row of the step-size probe
    int nb_col = 1, nb_row = 1;           // primal / dual SpMV kernels
    int nb_col_step = 1, nb_row_step = 1; // step-size variants (they write partials)
    int nb_res_col = 1, nb_res_row = 1;   // residual kernels
    int nb_m = 1, nb_nm = 1;              // elementwise kernels over m / n+m
};

static int valid_lanes(int g) { return g == 1 || g == 2 || g == 4 || g == 8 || g == 16 || g == 32; }

// The step-size probe gathers two vectors per entry (A x-bar and A dx), so it
// keeps the same requests in flight with twice the lanes of the row kernel
// (measured on B200 at 20 entries per row: 0.52 ms at 8 lanes vs 0.62 ms at 4).
static int probe_lanes(int g_row) { return g_row < 32 ? 2 * g_row : 32; }

// lanes option: 0 = lanes chosen by mean line length, 1..32 = lanes
template <class T>
Plan make_plan(const Ctx& ctx, int m, int n, long long nnz, int force_col, int force_row) {
    Plan p;
    const double mean_col = n > 0 ? (double)nnz / n : 1.0;
    const double mean_row = m > 0 ? (double)nnz / m : 1.0;
    p.g_col = valid_lanes(force_col) ? force_col : pick_lanes(mean_col);
    p.g_row = valid_lanes(force_row) ? force_row : pick_lanes(mean_row);
    p.g_probe = probe_lanes(p.g_row);
    MC_DISPATCH_G(p.g_col, {
        p.nb_col = grid_for(ctx, k_primal<G, false, T>, n, kBlock / G);
        p.nb_col_step = grid_for(ctx, k_primal<G, true, T>, n, kBlock / G);
    });
    MC_DISPATCH_G(p.g_row, p.nb_row = grid_for(ctx, k_dual<G, T>, m, kBlock / G));
    MC_DISPATCH_G(p.g_probe, p.nb_row_step = grid_for(ctx, k_dual_probe<G, T>, m, kBlock / G));
    MC_DISPATCH_G(p.g_col, p.nb_res_col = grid_for(ctx, k_residual_cols<G, T>, n, kBlock / G));
    MC_DISPATCH_G(p.g_row, p.nb_res_row = grid_for(ctx, k_residual_rows<G, T>, m, kBlock / G));
    p.nb_m = grid_for(ctx, k_dual_apply<T>, m, kBlock);
    p.nb_nm = grid_for(ctx, k_restart_copy<T>, (long long)n + m, kBlock);
    return p;
}

// ------------------------------------------------------------- transpose
// CSR(A) from CSC(A): count, scan, scatter, per-row sort (ascending column,
// so the layout and every SpMV over it are run-to-run deterministic).
// In-place inclusive scan of data[0..len), multi-level over tile totals; tmp
// holds (len + 1) / kScanTile + 4096 ints.
void inclusive_scan(Ctx& ctx, int* data, long long len, int* tmp, int kind = MC_KERNEL_SETUP) {
    cudaStream_t s = ctx.stream;
    std::vector<std::pair<int*, long long>> levels;
    while (true) {
        const long long tiles = (len + kScanTile - 1) / kScanTile;
        ctx.begin_launch(kind);
        k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, s>>>(data, len, tmp);
        ctx.end_launch();
        levels.push_back({data, len});
        if (tiles == 1) break;
        data = tmp;
        len = tiles;
        tmp += (tiles + 255) & ~255LL;
    }
    for (int l = (int)levels.size() - 2; l >= 0; --l) {
        const long long tiles = (levels[l].second + kScanTile - 1) / kScanTile;
        ctx.begin_launch(kind);
        k_scan_add<<<(unsigned)tiles, kBlock, 0, s>>>(levels[l].first, levels[l].second, levels[l + 1].first);
        ctx.end_launch();
    }
}

int build_csr(Ctx& ctx, int m, int n, long long nnz, const int* csc_start, const int* csc_row,
              const double* csc_val, int* csr_start, int* csr_col, double* csr_val, int* cursor,
              int* long_rows, int* counters /*[2]*/, int* scan_tmp) {
    cudaStream_t s = ctx.stream;
    CU(cudaMemsetAsync(csr_start, 0, sizeof(int) * (size_t)(m + 1), s));
    CU(cudaMemsetAsync(cursor, 0, sizeof(int) * (size_t)m, s));
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 2, s));
    if (nnz > 0) {
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_count_rows<<<blocks_for(ctx, nnz, kBlock) * 4, kBlock, 0, s>>>(nnz, csc_row, csr_start);
        ctx.end_launch();
    }
    inclusive_scan(ctx, csr_start, m + 1, scan_tmp);  // the m+1 counts
    if (nnz == 0) return ctx.launch_check("build_csr");
    const int nb_n = (int)((n + kBlock - 1) / kBlock);
    const int nb_m = (int)((m + kBlock - 1) / kBlock);
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_scatter_rows<<<nb_n, kBlock, 0, s>>>(n, csc_start, csc_row, csc_val, csr_start, cursor, csr_col, csr_val);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_sort_short_rows<<<nb_m, kBlock, 0, s>>>(m, csr_start, csr_col, csr_val, long_rows, counters);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_max_line<<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(m, csr_start, counters + 1);
    ctx.end_launch();
    int host_counters[2] = {0, 0};
    CU(cudaMemcpyAsync(host_counters, counters, sizeof host_counters, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    if (host_counters[0] > 0) {
        int* tmp_col = nullptr;
        double* tmp_val = nullptr;
        if (host_counters[1] > kSmemSortRow) {
            CU(cudaMallocAsync(reinterpret_cast<void**>(&tmp_col), sizeof(int) * (size_t)nnz, s));
            CU(cudaMallocAsync(reinterpret_cast<void**>(&tmp_val), sizeof(double) * (size_t)nnz, s));
        }
        const size_t smem = (size_t)kSmemSortRow * (sizeof(int) + sizeof(double));
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_sort_long_rows<<<host_counters[0], 1024, smem, s>>>(long_rows, csr_start, csr_col, csr_val, tmp_col, tmp_val);
        ctx.end_launch();
        if (tmp_col) {
            CU(cudaFreeAsync(tmp_col, s));
            CU(cudaFreeAsync(tmp_val, s));
        }
    }
    return ctx.launch_check("build_csr");
}

// ------------------------------------------------------------------ Ruiz
int ruiz(Ctx& ctx, int m, int n, long long nnz, const int* csc_start, const int* csc_row, double* csc_val,
         const int* csr_start, const int* csr_col, double* csr_val, double* row_scale, double* col_scale,
         double* r_tmp, double* c_tmp, double* partials, DevState* st, long long passes,
         double tolerance = 1e-3) {
    cudaStream_t s = ctx.stream;
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_fill<double><<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(row_scale, m, 1.0);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_fill<double><<<blocks_for(ctx, n, kBlock), kBlock, 0, s>>>(col_scale, n, 1.0);
    ctx.end_launch();
    if (nnz == 0) return ctx.launch_check("ruiz");
    const int nbc = blocks_for(ctx, n, kBlock), nbr = blocks_for(ctx, m, kBlock);
    for (long long pass = 0; pass < passes; ++pass) {
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_line_max<<<nbc, kBlock, 0, s>>>(n, csc_start, csc_val, c_tmp, partials + SLOT_A * kMaxPartials, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_line_max<<<nbr, kBlock, 0, s>>>(m, csr_start, csr_val, r_tmp, partials + SLOT_B * kMaxPartials, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_check<<<1, 1024, 0, s>>>(partials + SLOT_B * kMaxPartials, nbr, partials + SLOT_A * kMaxPartials,
                                        nbc, tolerance, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_deltas<<<nbr, kBlock, 0, s>>>(m, r_tmp, row_scale, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_deltas<<<nbc, kBlock, 0, s>>>(n, c_tmp, col_scale, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_rescale<<<nbc, kBlock, 0, s>>>(n, csc_start, csc_row, csc_val, c_tmp, r_tmp, 0, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_ruiz_rescale<<<nbr, kBlock, 0, s>>>(m, csr_start, csr_col, csr_val, r_tmp, c_tmp, 1, st);
        ctx.end_launch();
    }
    return ctx.launch_check("ruiz");
}

// ------------------------------------------------------- iteration chunks
// One precision's way of enqueuing iterations and restart checks.  FP64 runs
// the fused kernels on the iterate itself; the mixed form runs the FP32
// kernels on the correction and checks in FP64 (mixed.cuh).
struct Engine64 {
    // one launch shape per solve (the batch engines vary theirs)
    int shape_class(const DevState&) const { return 0; }
    void use_class(int) const {}

    Iterates<double> P;
    Original O;
    Plan pl;

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) {
            MC_DISPATCH_G(pl.g_col, (k_primal<G, true, double><<<pl.nb_col_step, kBlock, 0, s>>>(P, k)));
        } else {
            MC_DISPATCH_G(pl.g_col, (k_primal<G, false, double><<<pl.nb_col, kBlock, 0, s>>>(P, k)));
        }
        ctx.end_launch();
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            MC_DISPATCH_G(pl.g_probe, (k_dual_probe<G, double><<<pl.nb_row_step, kBlock, 0, s>>>(P)));
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            k_step_size<<<1, 1024, 0, s>>>(P.partials, pl.nb_col_step, pl.nb_row_step, P.st, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            k_dual_apply<double><<<pl.nb_m, kBlock, 0, s>>>(P, k);
            ctx.end_launch();
        } else {
            ctx.begin_launch(MC_KERNEL_DUAL);
            MC_DISPATCH_G(pl.g_row, (k_dual<G, double><<<pl.nb_row, kBlock, 0, s>>>(P, k)));
            ctx.end_launch();
        }
        return ctx.launch_check("iteration");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf& tr) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(pl.g_row, (k_residual_rows<G, double><<<pl.nb_res_row, kBlock, 0, s>>>(P, O)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(pl.g_col, (k_residual_cols<G, double><<<pl.nb_res_col, kBlock, 0, s>>>(P, O)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        k_finalize<<<1, 1024, 0, s>>>(P.partials, pl.nb_res_row, pl.nb_res_col, span, final_pass, O.offset, ctl, tr,
                                      P.st);
        ctx.end_launch();
        if (!final_pass) {
            ctx.begin_launch(MC_KERNEL_OTHER);
            k_restart_copy<double><<<pl.nb_nm, kBlock, 0, s>>>(P);
            ctx.end_launch();
        }
        return ctx.launch_check("check");
    }
};

struct EngineMixed {
    // one launch shape per solve (the batch engines vary theirs)
    int shape_class(const DevState&) const { return 0; }
    void use_class(int) const {}

    Iterates<float> P;
    MixedState M;
    Original O;
    Plan pl;
    int nb_res_row = 1, nb_res_col = 1, nb_recenter = 1, nb_apply = 1;

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) {
            MC_DISPATCH_G(pl.g_col, (k_primal<G, true, float><<<pl.nb_col_step, kBlock, 0, s>>>(P, k)));
        } else {
            MC_DISPATCH_G(pl.g_col, (k_primal<G, false, float><<<pl.nb_col, kBlock, 0, s>>>(P, k)));
        }
        ctx.end_launch();
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            MC_DISPATCH_G(pl.g_probe, (k_dual_probe<G, float><<<pl.nb_row_step, kBlock, 0, s>>>(P)));
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            k_step_size<<<1, 1024, 0, s>>>(P.partials, pl.nb_col_step, pl.nb_row_step, P.st, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            k_dual_apply_mx<<<nb_apply, kBlock, 0, s>>>(P, M, k);
            ctx.end_launch();
        } else {
            ctx.begin_launch(MC_KERNEL_DUAL);
            MC_DISPATCH_G(pl.g_row, (k_dual_mx<G><<<pl.nb_row, kBlock, 0, s>>>(P, M, k)));
            ctx.end_launch();
        }
        return ctx.launch_check("iteration (mixed)");
    }

    int residual_pass(Ctx& ctx) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(pl.g_row, (k_residual_rows_mx<G><<<nb_res_row, kBlock, 0, s>>>(P, M, O)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(pl.g_col, (k_residual_cols_mx<G><<<nb_res_col, kBlock, 0, s>>>(P, M, O)));
        ctx.end_launch();
        return ctx.launch_check("residual (mixed)");
    }

    int recenter(Ctx& ctx, int force) const {
        ctx.begin_launch(MC_KERNEL_OTHER);
        k_recenter_mx<<<nb_recenter, kBlock, 0, ctx.stream>>>(P, M, force);
        ctx.end_launch();
        return ctx.launch_check("recenter (mixed)");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf& tr) const {
        TRY(residual_pass(ctx));
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        k_finalize<<<1, 1024, 0, ctx.stream>>>(P.partials, nb_res_row, nb_res_col, span, final_pass, O.offset, ctl,
                                               tr, P.st);
        ctx.end_launch();
        if (!final_pass) TRY(recenter(ctx, 0));
        return ctx.launch_check("check (mixed)");
    }
};

// iterations [k0, k1) of the chunk that starts at global iteration `base`
template <class E>
int enqueue_span(Ctx& ctx, const E& eng, long long base, int k0, int k1, const Controls& ctl) {
    for (int k = k0; k < k1; ++k) {
        const bool step = ctl.adaptive_step && ((base + k) % 10 == 0);
        TRY(eng.iteration(ctx, k, step, ctl));
    }
    return MC_OK;
}

// Capture one full chunk (restart_every iterations + check) as a graph; the
// schedule of step-size iterations depends only on base % 10.
template <class E>
int chunk_graph(Ctx& ctx, const E& eng, long long base, long long R, const Controls& ctl, const TraceBuf& tr,
                int key, cudaGraphExec_t* out, long long recipe[MC_KERNEL_KINDS]) {
    long long before[MC_KERNEL_KINDS];
    std::memcpy(before, ctx.launches, sizeof before);
    CU(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
    ctx.capturing = true;
    int rc = enqueue_span(ctx, eng, base, 0, (int)R, ctl);
    if (rc == MC_OK) rc = eng.check(ctx, R, 0, ctl, tr);
    ctx.capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx.stream, &g);
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
        recipe[q] = ctx.launches[q] - before[q];
        ctx.launches[q] = before[q];
    }
    if (rc != MC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __LINE__);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e2 = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaGraphInstantiate", __LINE__);
    ctx.graphs[key] = exec;
    *out = exec;
    return MC_OK;
}

// Progress of the PDHG loop (pdlp.cpp:194-275) over restart chunks; kept
// between calls so that a solve can be driven a few chunks at a time.
struct ChunkLoop {
    long long full_chunks = 0;  // whole chunks within max_iterations
    long long chunk = 0;        // chunks enqueued so far
    long long base = 0;         // global iteration at the start of the next chunk
    bool done = false;          // a terminal status was seen by a poll
    bool have_prev = false;     // a poll is in flight
    int inflight = 0, ev_idx = 0;
    int cls = 0;                // the engine's launch-shape class, from the last poll
    long long recipe[40][MC_KERNEL_KINDS] = {};
};

// Enqueue up to `max_chunks` further chunks (each a CUDA graph replay), the
// host polling the device state one chunk group behind, so that the GPU never
// idles between chunks.  Returns with the stream synchronised and the state
// of the last chunk in ctx.h_state[2].
template <class E>
int loop_chunks(Ctx& ctx, const E& eng, DevState* st, ChunkLoop& L, long long max_chunks, long long R,
                int poll_every, const Controls& ctl, const TraceBuf& tr) {
    cudaStream_t s = ctx.stream;
    const long long stop = L.chunk + std::min(max_chunks, L.full_chunks - L.chunk);
    for (; L.chunk < stop && !L.done; ++L.chunk) {
        eng.use_class(L.cls);
        if (ctx.profiling) {
            TRY(enqueue_span(ctx, eng, L.base, 0, (int)R, ctl));
            TRY(eng.check(ctx, R, 0, ctl, tr));
            TRY(ctx.drain_profile());
        } else {
            // graphs keyed by the step-size phase (base % 10) and the class
            const int key = (int)(L.base % 10) + 10 * L.cls;
            auto it = ctx.graphs.find(key);
            cudaGraphExec_t exec = nullptr;
            if (it == ctx.graphs.end()) {
                TRY(chunk_graph(ctx, eng, L.base, R, ctl, tr, key, &exec, L.recipe[key]));
            } else {
                exec = it->second;
            }
            CU(cudaGraphLaunch(exec, s));
            for (int q = 0; q < MC_KERNEL_KINDS; ++q) ctx.launches[q] += L.recipe[key][q];
        }
        L.base += R;
        ++L.inflight;
        if (L.inflight >= poll_every || L.chunk + 1 == stop) {
            if (L.have_prev) {
                CU(cudaEventSynchronize(ctx.ev_poll[L.ev_idx ^ 1]));
                if (ctx.h_state[L.ev_idx ^ 1].done) L.done = true;
                L.cls = eng.shape_class(ctx.h_state[L.ev_idx ^ 1]);
            }
            CU(cudaMemcpyAsync(&ctx.h_state[L.ev_idx], st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
            CU(cudaEventRecord(ctx.ev_poll[L.ev_idx], s));
            L.have_prev = true;
            L.ev_idx ^= 1;
            L.inflight = 0;
        }
    }
    CU(cudaStreamSynchronize(s));
    CU(cudaMemcpy(&ctx.h_state[2], st, sizeof(DevState), cudaMemcpyDeviceToHost));
    L.have_prev = false;  // everything enqueued has completed
    L.inflight = 0;
    if (ctx.h_state[2].done) L.done = true;
    return MC_OK;
}

// After the last whole chunk: the remaining partial chunk, then the final
// evaluation (pdlp.cpp:263-265); after a whole number of chunks the last
// check already holds the averages' residuals.
template <class E>
int finish_chunks(Ctx& ctx, const E& eng, const ChunkLoop& L, long long maxit, long long R, const Controls& ctl,
                  const TraceBuf& tr) {
    if (!L.done && L.chunk == L.full_chunks) {
        const long long rem = maxit - L.full_chunks * R;
        if (rem > 0 || L.full_chunks == 0) {
            TRY(enqueue_span(ctx, eng, L.base, 0, (int)rem, ctl));
            TRY(eng.check(ctx, rem, 1, ctl, tr));
            TRY(ctx.drain_profile());
        }
    }
    CU(cudaStreamSynchronize(ctx.stream));
    return MC_OK;
}

// The whole PDHG loop (pdlp.cpp:194-275); returns with the stream synchronised.
template <class E>
int run_chunks(Ctx& ctx, const E& eng, DevState* st, long long maxit, long long R, int poll_every,
               const Controls& ctl, const TraceBuf& tr) {
    ctx.release_graphs();
    ChunkLoop L;
    L.full_chunks = maxit / R;
    TRY(loop_chunks(ctx, eng, st, L, L.full_chunks, R, poll_every, ctl, tr));
    return finish_chunks(ctx, eng, L, maxit, R, ctl, tr);
}

// Start selection.  `start(warm)` writes the starting point and resets the
// device state; `init()` finishes the engine-specific preparation.  With the
// guard, the reference's KKT score (max of primal, dual, gap; pdlp.cpp:133)
// of the warm start and of the cold start are evaluated on the device and the
// solve runs from the smaller.
template <class E, class Start, class Init>
int choose_start(Ctx& ctx, const E& eng, DevState* st, const Controls& ctl, bool have_warm, bool guard,
                 Start&& start, Init&& init, mc_pdlp_result* res) {
    TRY(init());
    res->warm_start_used = have_warm ? 1 : 0;
    if (!have_warm || !guard) return MC_OK;
    const TraceBuf none{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    auto score = [&](double* out) -> int {
        TRY(eng.check(ctx, 0, 1, ctl, none));
        CU(cudaMemcpyAsync(&ctx.h_state[1], st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx.stream));
        CU(cudaStreamSynchronize(ctx.stream));
        TRY(ctx.drain_profile());
        *out = ctx.h_state[1].nonfinite ? INFINITY : ctx.h_state[1].score;
        return MC_OK;
    };
    double sw = 0.0, s0 = 0.0;
    TRY(score(&sw));
    TRY(start(false));
    TRY(init());
    TRY(score(&s0));
    const bool use_warm = sw < s0;
    TRY(start(use_warm));
    TRY(init());
    res->warm_start_used = use_warm ? 1 : 0;
    res->warm_start_score = sw;
    res->cold_start_score = s0;
    return MC_OK;
}

// ------------------------------------------------------------------ solve
static void fill_message(mc_pdlp_result* r, const char* msg) {
    std::snprintf(r->message, sizeof r->message, "%s", msg);
}

int validate_options(const mc_pdlp_options* o) {
    if (!o) return set_error(MC_ERR_INVALID_ARGUMENT, "options is NULL");
    if (o->backend != MC_BACKEND_GPU)
        return set_error(MC_ERR_INVALID_ARGUMENT,
                         "backend must be MC_BACKEND_GPU: this engine has no CPU path");
    if (o->restart_every <= 0) return set_error(MC_ERR_INVALID_ARGUMENT, "restart_every must be positive");
    if (o->max_iterations < 0) return set_error(MC_ERR_INVALID_ARGUMENT, "max_iterations must be >= 0");
    if (o->restart_every > (1 << 20))
        return set_error(MC_ERR_INVALID_ARGUMENT, "restart_every above 2^20 is not supported");
    if (o->ruiz_iterations < 0) return set_error(MC_ERR_INVALID_ARGUMENT, "ruiz_iterations must be >= 0");
    if (!(o->restart_strategy >= 0 && o->restart_strategy <= 2))
        return set_error(MC_ERR_INVALID_ARGUMENT, "unknown restart_strategy %d", o->restart_strategy);
    if (o->precision != MC_PRECISION_FP64 && o->precision != MC_PRECISION_FP32_REFINE)
        return set_error(MC_ERR_INVALID_ARGUMENT, "unknown precision %d", o->precision);
    if ((o->lanes_per_column && !valid_lanes(o->lanes_per_column)) ||
        (o->lanes_per_row && !valid_lanes(o->lanes_per_row)))
        return set_error(MC_ERR_INVALID_ARGUMENT, "lanes per line must be 0 or a power of two <= 32");
    return MC_OK;
}

int validate_lp(const mc_lp* lp) {
    if (!lp) return set_error(MC_ERR_INVALID_ARGUMENT, "lp is NULL");
    if (lp->num_rows < 0 || lp->num_cols < 0 || lp->nnz < 0)
        return set_error(MC_ERR_INVALID_ARGUMENT, "negative dimension");
    if (lp->nnz >= (1LL << 31) - 1)
        return set_error(MC_ERR_RESOURCE_LIMIT, "nnz %lld exceeds the int32 index range", (long long)lp->nnz);
    if (lp->memory != MC_MEMORY_HOST && lp->memory != MC_MEMORY_DEVICE)
        return set_error(MC_ERR_INVALID_ARGUMENT, "unknown memory kind %d", lp->memory);
    if (lp->num_rows == 0 || lp->num_cols == 0) return MC_OK;
    if (!lp->col_start || (lp->nnz > 0 && (!lp->row_index || !lp->value)) || !lp->objective ||
        !lp->var_lower || !lp->var_upper || !lp->row_lower || !lp->row_upper)
        return set_error(MC_ERR_INVALID_ARGUMENT, "NULL array in lp");
    if (lp->memory == MC_MEMORY_HOST) {
        // cheap host checks first: the device validation re-checks everything
        if (lp->col_start[0] != 0 || (long long)lp->col_start[lp->num_cols] != lp->nnz)
            return set_error(MC_ERR_INVALID_ARGUMENT, "CSC terminal pointer mismatch");
    }
    return MC_OK;
}

// A solve in progress: what the PDHG loop and the output stage need between
// the calls of a stepwise solve (mc_pdlp_ctx_begin / _iterate / _finish).
struct Session {
    bool trivial = false, mixed = false, dev_in = false;
    Engine64 e64{};
    EngineMixed emx{};
    DevState* st = nullptr;
    Controls ctl{};
    TraceBuf tr{};
    mc_pdlp_trace* trace = nullptr;
    mc_pdlp_options o{};
    int m = 0, n = 0, poll_every = 1;
    ChunkLoop loop;
    double* x = nullptr;  // FP64 iterate (the mixed form's base point)
    double* y = nullptr;
    double* x_avg = nullptr;
    double* y_avg = nullptr;
    float* fx_avg = nullptr;  // mixed form: averaged corrections
    float* fy_avg = nullptr;
    double* col_scale = nullptr;
    double* row_scale = nullptr;
    double* x_stage = nullptr;
    double* y_stage = nullptr;
    double t_begin = 0.0;
    mc_pdlp_result head{};  // warm-start fields set at the start
};

void free_session(Session* s) { delete s; }

// Everything of a solve up to the first iteration (pdlp.cpp:139-191):
// uploads, validation, transpose, Ruiz, norms, start point.  The session is
// kept in the context until finish_session() or the next solve.
int begin_session(Ctx& ctx, const mc_lp* lp, const mc_pdlp_options* o, const double* warm_x,
                  const double* warm_y, mc_pdlp_trace* trace) {
    ctx.drop_session();
    const double t_begin = now_ms();
    if (trace) trace->count = 0;
    TRY(validate_options(o));
    TRY(validate_lp(lp));
    Session* S_ = new (std::nothrow) Session();
    if (!S_) return set_error(MC_ERR_OUT_OF_MEMORY, "host allocation failed");
    ctx.session = S_;
    Session& SS = *S_;
    SS.t_begin = t_begin;
    SS.o = *o;
    SS.trace = trace;
    mc_pdlp_result* res = &SS.head;
    const int m = lp->num_rows, n = lp->num_cols;
    const long long nnz = lp->nnz;
    SS.m = m;
    SS.n = n;
    if (m == 0 || n == 0) {  // pdlp.cpp:144-149
        SS.trivial = true;
        return MC_OK;
    }
    const bool mixed = o->precision == MC_PRECISION_FP32_REFINE;
    const bool dev_in = lp->memory == MC_MEMORY_DEVICE;
    SS.mixed = mixed;
    SS.dev_in = dev_in;
    cudaStream_t s = ctx.stream;
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
        ctx.launches[q] = 0;
        ctx.kernel_ms[q] = 0.0;
    }
    ctx.profiling = o->profile_kernels != 0;
    ctx.pending.clear();
    ctx.prof_used = 0;
    ctx.release_graphs();

    // ---- arena layout
    const long long trace_cap = trace ? trace->capacity : 0;
    Layout L;
    // structure and values are always copied (the matrix arrays padded by 16
    // entries so that 16-byte tile copies may overrun nnz)
    const size_t o_csc_start = L.add<int>(n + 1);
    const size_t o_csc_row = L.add<int>(nnz + 16);
    const size_t o_csc_val = L.add<double>(nnz + 16);
    const size_t o_csr_start = L.add<int>(m + 1);
    const size_t o_csr_col = L.add<int>(nnz + 16);
    const size_t o_csr_val = L.add<double>(nnz + 16);
    const size_t o_cursor = L.add<int>(m);
    const size_t o_long = L.add<int>(m);
    const size_t o_counters = L.add<int>(4);
    const size_t o_scan = L.add<int>((m + 1) / kScanTile + 4096);
    const size_t o_in_obj = dev_in ? 0 : L.add<double>(n);
    const size_t o_in_lo = dev_in ? 0 : L.add<double>(n);
    const size_t o_in_hi = dev_in ? 0 : L.add<double>(n);
    const size_t o_in_rlo = dev_in ? 0 : L.add<double>(m);
    const size_t o_in_rhi = dev_in ? 0 : L.add<double>(m);
    const size_t o_warm_x = (!dev_in && warm_x) ? L.add<double>(n) : 0;
    const size_t o_warm_y = (!dev_in && warm_y) ? L.add<double>(m) : 0;
    size_t o_n[14], o_m[12];
    for (auto& v : o_n) v = L.add<double>(n);
    for (auto& v : o_m) v = L.add<double>(m);
    const size_t o_partials = L.add<double>((long long)NUM_SLOTS * kMaxPartials);
    const size_t o_state = L.add<DevState>(1);
    // (x-bar, dx) pairs of the step-size iterations, in the iterate type
    const size_t o_xdx = mixed ? L.add<float>(2LL * n) : L.add<double>(2LL * n);
    const size_t o_tr_it = L.add<long long>(trace_cap);
    size_t o_tr[5];
    for (auto& v : o_tr) v = L.add<double>(trace_cap);
    const size_t o_tr_rs = L.add<int>(trace_cap);
    // mixed form: FP32 matrix copies, FP32 correction iterates and cycle data
    size_t o_f_cscv = 0, o_f_csrv = 0, o_fn[9] = {}, o_fm[8] = {};
    if (mixed) {
        o_f_cscv = L.add<float>(nnz + 16);
        o_f_csrv = L.add<float>(nnz + 16);
        for (auto& v : o_fn) v = L.add<float>(n);
        for (auto& v : o_fm) v = L.add<float>(m);
    }
    TRY(ctx.arena.reserve(L.offset));
    char* A = static_cast<char*>(ctx.arena.base);
    auto at = [&](size_t off) { return static_cast<void*>(A + off); };

    const int* csc_start = static_cast<int*>(at(o_csc_start));
    const int* csc_row = static_cast<int*>(at(o_csc_row));
    double* csc_val = static_cast<double*>(at(o_csc_val));
    int* csr_start = static_cast<int*>(at(o_csr_start));
    int* csr_col = static_cast<int*>(at(o_csr_col));
    double* csr_val = static_cast<double*>(at(o_csr_val));
    const double* in_obj = dev_in ? lp->objective : static_cast<double*>(at(o_in_obj));
    const double* in_lo = dev_in ? lp->var_lower : static_cast<double*>(at(o_in_lo));
    const double* in_hi = dev_in ? lp->var_upper : static_cast<double*>(at(o_in_hi));
    const double* in_rlo = dev_in ? lp->row_lower : static_cast<double*>(at(o_in_rlo));
    const double* in_rhi = dev_in ? lp->row_upper : static_cast<double*>(at(o_in_rhi));
    const double* d_warm_x = warm_x ? (dev_in ? warm_x : static_cast<double*>(at(o_warm_x))) : nullptr;
    const double* d_warm_y = warm_y ? (dev_in ? warm_y : static_cast<double*>(at(o_warm_y))) : nullptr;
    double* c = static_cast<double*>(at(o_n[0]));
    double* lo = static_cast<double*>(at(o_n[1]));
    double* hi = static_cast<double*>(at(o_n[2]));
    double* c_orig = static_cast<double*>(at(o_n[3]));
    double* lo_orig = static_cast<double*>(at(o_n[4]));
    double* hi_orig = static_cast<double*>(at(o_n[5]));
    double* col_norm = static_cast<double*>(at(o_n[6]));
    double* col_scale = static_cast<double*>(at(o_n[7]));
    double* x = static_cast<double*>(at(o_n[8]));
    double* x_bar = static_cast<double*>(at(o_n[9]));
    double* x_avg = static_cast<double*>(at(o_n[10]));
    double* dx = static_cast<double*>(at(o_n[11]));
    double* x_stage = static_cast<double*>(at(o_n[12]));
    double* blo = static_cast<double*>(at(o_m[0]));
    double* bhi = static_cast<double*>(at(o_m[1]));
    double* blo_orig = static_cast<double*>(at(o_m[2]));
    double* bhi_orig = static_cast<double*>(at(o_m[3]));
    double* row_norm = static_cast<double*>(at(o_m[4]));
    double* row_scale = static_cast<double*>(at(o_m[5]));
    double* y = static_cast<double*>(at(o_m[6]));
    double* y_avg = static_cast<double*>(at(o_m[7]));
    double* ax_bar = static_cast<double*>(at(o_m[8]));
    double* y_stage = static_cast<double*>(at(o_m[9]));
    double* partials = static_cast<double*>(at(o_partials));
    DevState* st = static_cast<DevState*>(at(o_state));

    // ---- uploads
    CU(cudaEventRecord(ctx.ev_a, s));
    const cudaMemcpyKind in_kind = dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CU(cudaMemcpyAsync(at(o_csc_start), lp->col_start, sizeof(int) * (size_t)(n + 1), in_kind, s));
    if (nnz) CU(cudaMemcpyAsync(at(o_csc_row), lp->row_index, sizeof(int) * (size_t)nnz, in_kind, s));
    CU(cudaMemsetAsync(static_cast<int*>(at(o_csc_row)) + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(static_cast<double*>(at(o_csc_val)) + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(static_cast<int*>(at(o_csr_col)) + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(static_cast<double*>(at(o_csr_val)) + nnz, 0, sizeof(double) * 16, s));
    if (!dev_in) {
        CU(cudaMemcpyAsync(at(o_in_obj), lp->objective, sizeof(double) * (size_t)n, in_kind, s));
        CU(cudaMemcpyAsync(at(o_in_lo), lp->var_lower, sizeof(double) * (size_t)n, in_kind, s));
        CU(cudaMemcpyAsync(at(o_in_hi), lp->var_upper, sizeof(double) * (size_t)n, in_kind, s));
        CU(cudaMemcpyAsync(at(o_in_rlo), lp->row_lower, sizeof(double) * (size_t)m, in_kind, s));
        CU(cudaMemcpyAsync(at(o_in_rhi), lp->row_upper, sizeof(double) * (size_t)m, in_kind, s));
        if (warm_x) CU(cudaMemcpyAsync(at(o_warm_x), warm_x, sizeof(double) * (size_t)n, in_kind, s));
        if (warm_y) CU(cudaMemcpyAsync(at(o_warm_y), warm_y, sizeof(double) * (size_t)m, in_kind, s));
    }
    if (nnz) CU(cudaMemcpyAsync(csc_val, lp->value, sizeof(double) * (size_t)nnz, in_kind, s));
    CU(cudaEventRecord(ctx.ev_b, s));

    // ---- validation (every later gather depends on it)
    int* counters = static_cast<int*>(at(o_counters));
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, csc_start, csc_row, csc_val, counters + 2);
    ctx.end_launch();
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    if (bad) {
        return set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix (%s%s%s%s)",
                         (bad & 1) ? "column pointers " : "", (bad & 2) ? "row index out of range " : "",
                         (bad & 4) ? "rows not strictly increasing " : "",
                         (bad & 8) ? "zero or non-finite value" : "");
    }

    // ---- setup (FP64, both forms)
    CU(cudaMemsetAsync(st, 0, sizeof(DevState), s));
    TRY(build_csr(ctx, m, n, nnz, csc_start, csc_row, csc_val, csr_start, csr_col, csr_val,
                  static_cast<int*>(at(o_cursor)), static_cast<int*>(at(o_long)), counters,
                  static_cast<int*>(at(o_scan))));
    TRY(ruiz(ctx, m, n, nnz, csc_start, csc_row, csc_val, csr_start, csr_col, csr_val, row_scale, col_scale,
             ax_bar, dx, partials, st, o->ruiz_scaling ? o->ruiz_iterations : 0));
    const double obj_sign = (lp->objective_sense == MC_MAXIMIZE) ? -1.0 : 1.0;
    const int nbc = blocks_for(ctx, n, kBlock), nbr = blocks_for(ctx, m, kBlock);
    // starting point (pdlp.cpp:153-191): warm = the caller's warm start and
    // primal weight, cold = x = proj(0), y = 0 and the derived weight
    auto start = [&](bool warm) -> int {
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_setup_cols<<<nbc, kBlock, 0, s>>>(n, csc_start, csc_val, in_obj, in_lo, in_hi, col_scale,
                                            warm ? d_warm_x : nullptr, obj_sign, c, lo, hi, c_orig, lo_orig,
                                            hi_orig, col_norm, x, x_avg, partials);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_setup_rows<<<nbr, kBlock, 0, s>>>(m, csr_start, csr_val, in_rlo, in_rhi, row_scale,
                                            warm ? d_warm_y : nullptr, blo, bhi, blo_orig, bhi_orig, row_norm, y,
                                            y_avg, partials);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_setup_scalars<<<1, 1024, 0, s>>>(partials, nbc, nbr,
                                           (warm || !o->warm_start_guard) ? o->initial_primal_weight : 0.0,
                                           o->step_size_reduction, st);
        ctx.end_launch();
        return ctx.launch_check("setup");
    };
    const bool have_warm = d_warm_x != nullptr || d_warm_y != nullptr;
    TRY(start(have_warm));

    Original O{c_orig, in_obj, lo_orig, hi_orig, blo_orig, bhi_orig, col_scale, row_scale, lp->objective_offset};
    Controls ctl{o->primal_tolerance, o->dual_tolerance, o->gap_tolerance, o->restart_reduction_factor,
                 o->primal_weight_smoothing, o->restart_every, o->restart_strategy, o->adaptive_step_size,
                 o->adaptive_primal_weight};
    TraceBuf tr{trace_cap, static_cast<long long*>(at(o_tr_it)), static_cast<double*>(at(o_tr[0])),
                static_cast<double*>(at(o_tr[1])), static_cast<double*>(at(o_tr[2])),
                static_cast<double*>(at(o_tr[3])), static_cast<double*>(at(o_tr[4])),
                static_cast<int*>(at(o_tr_rs))};
    const int poll_every = o->check_every_chunks > 0 ? o->check_every_chunks : 1;

    // ---- the PDHG engine of the chosen form
    float* fx_avg = nullptr;
    float* fy_avg = nullptr;
    if (!mixed) {
        Engine64& eng = SS.e64;
        Iterates<double>& P = eng.P;
        P.m = m;
        P.n = n;
        P.csc_start = csc_start;
        P.csc_row = csc_row;
        P.csc_val = csc_val;
        P.csr_start = csr_start;
        P.csr_col = csr_col;
        P.csr_val = csr_val;
        P.c = c;
        P.lo = lo;
        P.hi = hi;
        P.blo = blo;
        P.bhi = bhi;
        P.col_norm = col_norm;
        P.row_norm = row_norm;
        P.x = x;
        P.x_bar = x_bar;
        P.x_avg = x_avg;
        P.dx = dx;
        P.xdx = static_cast<double*>(at(o_xdx));
        P.y = y;
        P.y_avg = y_avg;
        P.ax_bar = ax_bar;
        P.partials = partials;
        P.st = st;
        eng.O = O;
        eng.pl = make_plan<double>(ctx, m, n, nnz, o->lanes_per_column, o->lanes_per_row);
        TRY(choose_start(ctx, eng, st, ctl, have_warm, o->warm_start_guard != 0, start, [] { return MC_OK; }, res));
    } else {
        EngineMixed& eng = SS.emx;
        float* f_cscv = static_cast<float*>(at(o_f_cscv));
        float* f_csrv = static_cast<float*>(at(o_f_csrv));
        float* f_g = static_cast<float*>(at(o_fn[0]));
        float* f_lo = static_cast<float*>(at(o_fn[1]));
        float* f_hi = static_cast<float*>(at(o_fn[2]));
        float* f_cn = static_cast<float*>(at(o_fn[3]));
        float* f_x = static_cast<float*>(at(o_fn[4]));
        float* f_xb = static_cast<float*>(at(o_fn[5]));
        float* f_xa = static_cast<float*>(at(o_fn[6]));
        float* f_dx = static_cast<float*>(at(o_fn[7]));
        float* f_rn = static_cast<float*>(at(o_fm[0]));
        float* f_y = static_cast<float*>(at(o_fm[1]));
        float* f_ya = static_cast<float*>(at(o_fm[2]));
        float* f_axb = static_cast<float*>(at(o_fm[3]));
        float* f_rlo = static_cast<float*>(at(o_fm[4]));
        float* f_rhi = static_cast<float*>(at(o_fm[5]));
        float* f_yb = static_cast<float*>(at(o_fm[6]));
        fx_avg = f_xa;
        fy_avg = f_ya;
        const int nbz = blocks_for(ctx, nnz + 16, kBlock) * 4;
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, csc_val, f_cscv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, csr_val, f_csrv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbc, kBlock, 0, s>>>(n, col_norm, f_cn);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbr, kBlock, 0, s>>>(m, row_norm, f_rn);
        ctx.end_launch();

        Iterates<float>& P = eng.P;
        P.m = m;
        P.n = n;
        P.csc_start = csc_start;
        P.csc_row = csc_row;
        P.csc_val = f_cscv;
        P.csr_start = csr_start;
        P.csr_col = csr_col;
        P.csr_val = f_csrv;
        P.c = f_g;
        P.lo = f_lo;
        P.hi = f_hi;
        P.blo = nullptr;  // the mixed dual step reads r_lo / r_hi instead
        P.bhi = nullptr;
        P.col_norm = f_cn;
        P.row_norm = f_rn;
        P.x = f_x;
        P.x_bar = f_xb;
        P.x_avg = f_xa;
        P.dx = f_dx;
        P.xdx = static_cast<float*>(at(o_xdx));
        P.y = f_y;
        P.y_avg = f_ya;
        P.ax_bar = f_axb;
        P.partials = partials;
        P.st = st;
        MixedState& M = eng.M;
        M.x_hat = x;  // the FP64 start point becomes the first base
        M.y_hat = y;
        M.ax_full = ax_bar;
        M.aty_full = dx;
        M.c64 = c;
        M.lo64 = lo;
        M.hi64 = hi;
        M.blo64 = blo;
        M.bhi64 = bhi;
        M.csc_val64 = csc_val;
        M.csr_val64 = csr_val;
        M.g = f_g;
        M.lo = f_lo;
        M.hi = f_hi;
        M.r_lo = f_rlo;
        M.r_hi = f_rhi;
        M.yb = f_yb;
        eng.O = O;
        eng.pl = make_plan<float>(ctx, m, n, nnz, o->lanes_per_column, o->lanes_per_row);
        // the FP32 dual kernel has no block partials: one block per kBlock/G rows
        // (about 40 waves) lets the block scheduler even out the last wave,
        // 13% faster on B200 than one resident wave; the FP64 and primal
        // kernels run slower that way and keep one wave
        eng.pl.nb_row = (int)std::max<long long>(1, ((long long)m + kBlock / eng.pl.g_row - 1) / (kBlock / eng.pl.g_row));
        MC_DISPATCH_G(eng.pl.g_row, eng.nb_res_row = grid_for(ctx, k_residual_rows_mx<G>, m, kBlock / G));
        MC_DISPATCH_G(eng.pl.g_col, eng.nb_res_col = grid_for(ctx, k_residual_cols_mx<G>, n, kBlock / G));
        eng.nb_recenter = grid_for(ctx, k_recenter_mx, (long long)n + m, kBlock);
        eng.nb_apply = grid_for(ctx, k_dual_apply_mx, m, kBlock);
        // the first correction LP around the start point (zero corrections)
        auto init = [&]() -> int {
            for (float* z : {f_x, f_xb, f_xa, f_dx}) CU(cudaMemsetAsync(z, 0, sizeof(float) * (size_t)n, s));
            for (float* z : {f_y, f_ya, f_axb}) CU(cudaMemsetAsync(z, 0, sizeof(float) * (size_t)m, s));
            TRY(eng.residual_pass(ctx));
            return eng.recenter(ctx, 1);
        };
        TRY(choose_start(ctx, eng, st, ctl, have_warm, o->warm_start_guard != 0, start, init, res));
    }
    SS.st = st;
    SS.ctl = ctl;
    SS.tr = tr;
    SS.poll_every = poll_every;
    SS.loop.full_chunks = o->max_iterations / o->restart_every;
    SS.x = x;
    SS.y = y;
    SS.x_avg = x_avg;
    SS.y_avg = y_avg;
    SS.fx_avg = fx_avg;
    SS.fy_avg = fy_avg;
    SS.col_scale = col_scale;
    SS.row_scale = row_scale;
    SS.x_stage = x_stage;
    SS.y_stage = y_stage;
    ctx.release_graphs();
    return MC_OK;
}

// Up to `chunks` further restart chunks of the session's PDHG loop (each
// restart_every iterations and the restart check, pdlp.cpp:194-262).
int iterate_session(Ctx& ctx, long long chunks, long long* iterations, int* finished) {
    Session* S = ctx.session;
    if (!S) return set_error(MC_ERR_INVALID_ARGUMENT, "no solve in progress on this context");
    if (chunks < 0) return set_error(MC_ERR_INVALID_ARGUMENT, "chunks must be >= 0");
    if (!S->trivial && chunks > 0) {
        const long long R = S->o.restart_every;
        if (S->mixed) TRY(loop_chunks(ctx, S->emx, S->st, S->loop, chunks, R, S->poll_every, S->ctl, S->tr));
        else TRY(loop_chunks(ctx, S->e64, S->st, S->loop, chunks, R, S->poll_every, S->ctl, S->tr));
    }
    if (iterations) *iterations = S->trivial ? 0 : S->loop.chunk * S->o.restart_every;
    if (finished) *finished = (S->trivial || S->loop.done || S->loop.chunk == S->loop.full_chunks) ? 1 : 0;
    if (S->loop.done && iterations && !S->trivial) *iterations = ctx.h_state[2].iter;
    return MC_OK;
}

// The end of a solve: the remaining partial chunk and final evaluation when
// the loop ran to max_iterations, then the unscaled averages (pdlp.cpp:263-276)
// and the result.  Ends the session.
int finish_session(Ctx& ctx, double* x_out, double* y_out, mc_pdlp_result* res) {
    Session* S = ctx.session;
    if (!S) return set_error(MC_ERR_INVALID_ARGUMENT, "no solve in progress on this context");
    if (!res) return set_error(MC_ERR_INVALID_ARGUMENT, "result is NULL");
    std::memcpy(res, &S->head, sizeof *res);
    std::snprintf(res->backend_actually_used, sizeof res->backend_actually_used, "cuda");
    res->certificate = MC_CERT_NONE;  // a single solve keeps the reference's statuses (no certificates)
    res->certificate_index = -1;
    const mc_pdlp_options* o = &S->o;
    if (S->trivial) {
        res->status = MC_PDLP_OPTIMAL;
        res->tolerance = o->primal_tolerance;
        fill_message(res, "trivial");
        res->total_ms = now_ms() - S->t_begin;
        ctx.drop_session();
        return MC_OK;
    }
    cudaStream_t s = ctx.stream;
    const int m = S->m, n = S->n;
    const bool mixed = S->mixed, dev_in = S->dev_in;
    const long long R = o->restart_every;
    if (mixed) TRY(finish_chunks(ctx, S->emx, S->loop, o->max_iterations, R, S->ctl, S->tr));
    else TRY(finish_chunks(ctx, S->e64, S->loop, o->max_iterations, R, S->ctl, S->tr));
    DevState* st = S->st;
    mc_pdlp_trace* trace = S->trace;
    const long long trace_cap = trace ? trace->capacity : 0;
    CU(cudaMemcpy(&ctx.h_state[2], st, sizeof(DevState), cudaMemcpyDeviceToHost));
    CU(cudaEventRecord(ctx.ev_c, s));

    // ---- outputs
    const bool dev_out = dev_in;
    double* xo = dev_out ? x_out : (x_out ? S->x_stage : nullptr);
    double* yo = dev_out ? y_out : (y_out ? S->y_stage : nullptr);
    if (xo || yo) {
        const int nb = blocks_for(ctx, (long long)n + m, kBlock);
        ctx.begin_launch(MC_KERNEL_OTHER);
        if (mixed)
            k_unscale_out_mx<<<nb, kBlock, 0, s>>>(n, m, S->x, S->fx_avg, S->y, S->fy_avg, S->col_scale,
                                                   S->row_scale, xo, yo);
        else k_unscale_out<<<nb, kBlock, 0, s>>>(n, m, S->x_avg, S->y_avg, S->col_scale, S->row_scale, xo, yo);
        ctx.end_launch();
        TRY(ctx.launch_check("unscale"));
    }
    cudaEvent_t ev_d2h = ctx.ev_d;
    CU(cudaEventRecord(ctx.ev_c, s));
    if (!dev_out) {
        if (x_out) CU(cudaMemcpyAsync(x_out, S->x_stage, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s));
        if (y_out) CU(cudaMemcpyAsync(y_out, S->y_stage, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaMemcpyAsync(&ctx.h_state[3], st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    CU(cudaEventRecord(ev_d2h, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    const DevState& DS = ctx.h_state[3];
    if (trace && trace_cap > 0) {
        const long long cnt = std::min<long long>(DS.checks, trace_cap);
        trace->count = cnt;
        const TraceBuf& tb = S->tr;
        if (cnt > 0) {
            CU(cudaMemcpy(trace->iteration, tb.iteration, sizeof(long long) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->primal_infeasibility, tb.primal, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->dual_infeasibility, tb.dual, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->duality_gap, tb.gap, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->step_size, tb.eta, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->primal_weight, tb.omega, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(trace->restarted, tb.restarted, sizeof(int) * cnt, cudaMemcpyDeviceToHost));
        }
    }
    float h2d = 0.f, kern = 0.f, d2h = 0.f;
    CU(cudaEventElapsedTime(&h2d, ctx.ev_a, ctx.ev_b));
    CU(cudaEventElapsedTime(&kern, ctx.ev_b, ctx.ev_c));
    CU(cudaEventElapsedTime(&d2h, ctx.ev_c, ev_d2h));
    res->status = DS.status;
    res->objective = DS.objective;
    res->primal_infeasibility = DS.primal_infeas;
    res->dual_infeasibility = DS.dual_infeas;
    res->duality_gap = DS.gap;
    res->tolerance = o->primal_tolerance;
    res->iterations = DS.iter;
    fill_message(res, DS.status == MC_PDLP_OPTIMAL ? "PDLP converged"
                      : DS.status == MC_PDLP_NUMERICAL_FAILURE ? "non-finite iterate or residual"
                                                              : "iteration limit reached");
    res->h2d_ms = dev_in ? 0.0 : h2d;
    res->kernel_ms = kern + (dev_in ? h2d : 0.0);
    res->d2h_ms = dev_out ? 0.0 : d2h;
    res->ruiz_iterations_executed = o->ruiz_scaling ? DS.ruiz_passes : 0;
    res->restarts = DS.restarts;
    res->final_primal_weight = DS.omega;
    res->final_step_size = DS.eta;
    res->refinement_rounds = mixed ? DS.restarts : 0;  // each restart re-centres the FP64 base
    res->inner_iterations = mixed ? DS.iter : 0;
    long long total = 0;
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
        res->launches_by_kind[q] = ctx.launches[q];
        res->kernel_ms_by_kind[q] = ctx.kernel_ms[q];
        total += ctx.launches[q];
    }
    res->kernel_launches = total;
    res->total_ms = now_ms() - S->t_begin;
    ctx.drop_session();
    return MC_OK;
}

int solve_lp(Ctx& ctx, const mc_lp* lp, const mc_pdlp_options* o, const double* warm_x,
             const double* warm_y, double* x_out, double* y_out, mc_pdlp_result* res,
             mc_pdlp_trace* trace) {
    if (!res) return set_error(MC_ERR_INVALID_ARGUMENT, "result is NULL");
    std::memset(res, 0, sizeof *res);
    std::snprintf(res->backend_actually_used, sizeof res->backend_actually_used, "cuda");
    int rc = begin_session(ctx, lp, o, warm_x, warm_y, trace);
    if (rc == MC_OK) rc = iterate_session(ctx, LLONG_MAX, nullptr, nullptr);
    if (rc == MC_OK) rc = finish_session(ctx, x_out, y_out, res);
    if (rc != MC_OK) ctx.drop_session();
    return rc;
}

}  // namespace mc
