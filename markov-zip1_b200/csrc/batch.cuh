// Host driver of the batched solve (included once, by engine.cu after solve.cuh).
#pragma once

#include "batch_kernels.cuh"
#include "solve.cuh"

#include <tuple>
#include <vector>

namespace mc {

// What both batched engines share: the work queue and the lanes.
struct BatchCommon {
    BatchRefs B;
    DevState* global = nullptr;  // poll flag: every LP done
    int* active = nullptr;       // the work queue (B.active, writable)
    int* active_count = nullptr;
    int* lp_offset = nullptr;    // [2 * (nlp + 1)] each LP's range in the queue
    int g_col = 1, g_row = 1;

    // persistent grids: one wave of resident blocks, at most one per tile, and
    // at most grid_cap blocks once few tiles are left running
    mutable int grid_cap = 1 << 30;
    template <class K>
    int grid(const Ctx& ctx, K kernel, int tiles) const {
        return std::min(grid_for(ctx, kernel, tiles, 1), grid_cap);
    }

    // Grid classes of the chunk loop: as LPs converge the polled count of
    // running tiles (an upper bound: it only falls) selects a chunk graph
    // whose persistent kernels launch fewer blocks, so the tail of a batch,
    // where a few slow LPs run on alone, pays for their tiles only.
    static constexpr int kClassCap[4] = {1 << 30, 512, 128, 32};
    int shape_class(const DevState& polled) const {
        const int active = std::max(polled.active_tiles[0], polled.active_tiles[1]);
        int c = 0;
        while (c + 1 < 4 && active <= kClassCap[c + 1]) ++c;
        return c;
    }
    void use_class(int c) const { grid_cap = kClassCap[c]; }

    int compact(Ctx& ctx) const {
        ctx.begin_launch(MC_KERNEL_OTHER);
        kb_compact<<<1, kCompactThreads, 0, ctx.stream>>>(B, lp_offset, active_count, global);
        ctx.end_launch();
        const int tiles = B.cols.ntiles + B.rows.ntiles;
        ctx.begin_launch(MC_KERNEL_OTHER);
        kb_fill_active<<<(tiles + kBlock - 1) / kBlock, kBlock, 0, ctx.stream>>>(B, lp_offset, active);
        ctx.end_launch();
        return MC_OK;
    }
};

// FP64 batched PDHG.
struct EngineBatch : BatchCommon {
    Iterates<double> P;
    Original O;

    int primal(Ctx& ctx, int g, bool step, int k) const {
        cudaStream_t s = ctx.stream;
        const int nc = B.cols.ntiles;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) {
            MC_DISPATCH_G(g, (kb_primal<G, true, double><<<grid(ctx, kb_primal<G, true, double>, nc), kBlock, 0, s>>>(P, B, k)));
        } else {
            MC_DISPATCH_G(g, (kb_primal<G, false, double><<<grid(ctx, kb_primal<G, false, double>, nc), kBlock, 0, s>>>(P, B, k)));
        }
        ctx.end_launch();
        return MC_OK;
    }

    int dual(Ctx& ctx, int g, int k) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_DUAL);
        MC_DISPATCH_G(g, (kb_dual<G><<<grid(ctx, kb_dual<G>, B.rows.ntiles), kBlock, 0, s>>>(P, B, k)));
        ctx.end_launch();
        return MC_OK;
    }

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        const int nr = B.rows.ntiles;
        TRY(primal(ctx, g_col, step, k));
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            MC_DISPATCH_G(probe_lanes(g_row), (kb_dual_probe<G, double><<<grid(ctx, kb_dual_probe<G, double>, nr), kBlock, 0, s>>>(P, B)));
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            kb_step_size<<<B.nlp, 256, 0, s>>>(P.partials, B, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kb_dual_apply<<<grid(ctx, kb_dual_apply, nr), kBlock, 0, s>>>(P, B, k);
            ctx.end_launch();
        } else {
            TRY(dual(ctx, g_row, k));
        }
        return ctx.launch_check("batch iteration");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf&) const {
        cudaStream_t s = ctx.stream;
        const int nc = B.cols.ntiles, nr = B.rows.ntiles;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_row, (kb_residual_rows<G><<<grid(ctx, kb_residual_rows<G>, nr), kBlock, 0, s>>>(P, O, B)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_col, (kb_residual_cols<G><<<grid(ctx, kb_residual_cols<G>, nc), kBlock, 0, s>>>(P, O, B)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kb_finalize<<<B.nlp, 256, 0, s>>>(P.partials, B, span, final_pass, ctl);
        ctx.end_launch();
        if (!final_pass) {
            ctx.begin_launch(MC_KERNEL_OTHER);
            kb_restart_copy<<<grid(ctx, kb_restart_copy, nc + nr), kBlock, 0, s>>>(P, B);
            ctx.end_launch();
        }
        TRY(compact(ctx));
        return ctx.launch_check("batch check");
    }
};

// FP32 + FP64-refinement batched PDHG (the mixed form of solve.cuh, per LP).
struct EngineBatchMixed : BatchCommon {
    Iterates<float> P;
    MixedState M;
    Original O;

    int primal(Ctx& ctx, int g, bool step, int k) const {
        cudaStream_t s = ctx.stream;
        const int nc = B.cols.ntiles;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) {
            MC_DISPATCH_G(g, (kb_primal<G, true, float><<<grid(ctx, kb_primal<G, true, float>, nc), kBlock, 0, s>>>(P, B, k)));
        } else {
            MC_DISPATCH_G(g, (kb_primal<G, false, float><<<grid(ctx, kb_primal<G, false, float>, nc), kBlock, 0, s>>>(P, B, k)));
        }
        ctx.end_launch();
        return MC_OK;
    }

    int dual(Ctx& ctx, int g, int k) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_DUAL);
        MC_DISPATCH_G(g, (kb_dual_mx<G><<<grid(ctx, kb_dual_mx<G>, B.rows.ntiles), kBlock, 0, s>>>(P, M, B, k)));
        ctx.end_launch();
        return MC_OK;
    }

    int residual_pass(Ctx& ctx) const {
        cudaStream_t s = ctx.stream;
        const int nc = B.cols.ntiles, nr = B.rows.ntiles;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_row, (kb_residual_rows_mx<G><<<grid(ctx, kb_residual_rows_mx<G>, nr), kBlock, 0, s>>>(P, M, O, B)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_col, (kb_residual_cols_mx<G><<<grid(ctx, kb_residual_cols_mx<G>, nc), kBlock, 0, s>>>(P, M, O, B)));
        ctx.end_launch();
        return ctx.launch_check("batch residual (mixed)");
    }

    int recenter(Ctx& ctx, int force) const {
        ctx.begin_launch(MC_KERNEL_OTHER);
        kb_recenter_mx<<<grid(ctx, kb_recenter_mx, B.cols.ntiles + B.rows.ntiles), kBlock, 0, ctx.stream>>>(P, M, B,
                                                                                                          force);
        ctx.end_launch();
        return ctx.launch_check("batch recenter (mixed)");
    }

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        const int nr = B.rows.ntiles;
        TRY(primal(ctx, g_col, step, k));
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            MC_DISPATCH_G(probe_lanes(g_row), (kb_dual_probe<G, float><<<grid(ctx, kb_dual_probe<G, float>, nr), kBlock, 0, s>>>(P, B)));
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            kb_step_size<<<B.nlp, 256, 0, s>>>(P.partials, B, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kb_dual_apply_mx<<<grid(ctx, kb_dual_apply_mx, nr), kBlock, 0, s>>>(P, M, B, k);
            ctx.end_launch();
        } else {
            TRY(dual(ctx, g_row, k));
        }
        return ctx.launch_check("batch iteration (mixed)");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf&) const {
        TRY(residual_pass(ctx));
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kb_finalize<<<B.nlp, 256, 0, ctx.stream>>>(P.partials, B, span, final_pass, ctl);
        ctx.end_launch();
        if (!final_pass) TRY(recenter(ctx, 0));
        TRY(compact(ctx));
        return ctx.launch_check("batch check (mixed)");
    }
};

// The autotuner: lanes per column for the A^T y kernel and lanes per row for
// the A x kernel, each chosen by timing that kernel over the batch itself at
// every power of two 1..32 (best of two timed launches after a warm one);
// then the block shape of the persistent kernels' work -- lines per tile, 1,
// 2 or 4 block-steps -- by timing both kernels at each (`retile(steps)`
// rebuilds the tile tables and the work queue).  Short tiles spread the few
// LPs that run late in a batch over many blocks; long tiles cut per-tile
// overhead when the LPs finish together.  It runs from the start iterate,
// which is saved first and put back after, so the solve that follows is the
// one the chosen shape gives.  The choice is kept per context, batch shape
// and precision: later solves of the same shape reuse it (and repeat
// bit-identically).
template <class E, class Retile>
int tune_lanes(Ctx& ctx, E& eng, int precision, void* const save_n[3], void* const save_m[2], Retile&& retile) {
    const auto key = std::make_tuple((long long)eng.P.n, (long long)eng.P.m, (long long)eng.B.nlp,
                                     (long long)eng.B.cols.ntiles * 4 + precision, (long long)eng.B.rows.ntiles);
    auto hit = ctx.lane_cache.find(key);
    if (hit != ctx.lane_cache.end()) {
        eng.g_col = std::get<0>(hit->second);
        eng.g_row = std::get<1>(hit->second);
        return retile(std::get<2>(hit->second));
    }
    cudaStream_t s = ctx.stream;
    const size_t elem = sizeof(*eng.P.x);
    const size_t bn = elem * (size_t)eng.P.n, bm = elem * (size_t)eng.P.m;
    void* const cur_n[3] = {eng.P.x, eng.P.x_bar, eng.P.x_avg};
    void* const cur_m[2] = {eng.P.y, eng.P.y_avg};
    for (int q = 0; q < 3; ++q) CU(cudaMemcpyAsync(save_n[q], cur_n[q], bn, cudaMemcpyDeviceToDevice, s));
    for (int q = 0; q < 2; ++q) CU(cudaMemcpyAsync(save_m[q], cur_m[q], bm, cudaMemcpyDeviceToDevice, s));
    auto ok = [](cudaError_t e, const char* what) { return e == cudaSuccess ? MC_OK : cuda_fail(e, what, __LINE__); };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU(cudaEventCreate(&e0));
    int rc = ok(cudaEventCreate(&e1), "cudaEventCreate");
    // best of two timed launches (after a warm one) of primal (which = 0),
    // dual (1) or both (2) at lanes g
    auto time_kernels = [&](int which, int g, float* out) -> int {
        float t_min = 3.0e38f;
        for (int rep = 0; rep < 3; ++rep) {
            float ms = 0.f;
            TRY(ok(cudaEventRecord(e0, s), "cudaEventRecord"));
            if (which != 1) TRY(eng.primal(ctx, which == 2 ? eng.g_col : g, false, 0));
            if (which != 0) TRY(eng.dual(ctx, which == 2 ? eng.g_row : g, 0));
            TRY(ctx.launch_check("autotuner"));
            TRY(ok(cudaEventRecord(e1, s), "cudaEventRecord"));
            TRY(ok(cudaEventSynchronize(e1), "cudaEventSynchronize"));
            TRY(ok(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime"));
            if (rep > 0 && ms < t_min) t_min = ms;
        }
        *out = t_min;
        return MC_OK;
    };
    float best[2] = {3.0e38f, 3.0e38f};
    int pick[2] = {eng.g_col, eng.g_row};
    for (int g = 1; g <= 32 && rc == MC_OK; g *= 2) {
        for (int which = 0; which < 2 && rc == MC_OK; ++which) {
            float t = 0.f;
            rc = time_kernels(which, g, &t);
            if (rc == MC_OK && t < best[which]) {
                best[which] = t;
                pick[which] = g;
            }
        }
    }
    eng.g_col = pick[0];
    eng.g_row = pick[1];
    int steps_pick = 1;
    float steps_best = 3.0e38f;
    for (int steps = 1; steps <= 4 && rc == MC_OK; steps *= 2) {
        float t = 0.f;
        rc = retile(steps);
        if (rc == MC_OK) rc = time_kernels(2, 0, &t);
        if (rc == MC_OK && t < steps_best) {
            steps_best = t;
            steps_pick = steps;
        }
    }
    if (rc == MC_OK) rc = retile(steps_pick);
    cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    TRY(rc);
    for (int q = 0; q < 3; ++q) CU(cudaMemcpyAsync(cur_n[q], save_n[q], bn, cudaMemcpyDeviceToDevice, s));
    for (int q = 0; q < 2; ++q) CU(cudaMemcpyAsync(cur_m[q], save_m[q], bm, cudaMemcpyDeviceToDevice, s));
    ctx.lane_cache[key] = std::make_tuple(pick[0], pick[1], steps_pick);
    return MC_OK;
}

// Tiles of `per_tile` lines that never cross an LP boundary.
static void make_tiles(const std::vector<long long>& off, int per_tile, std::vector<int>& lp, std::vector<int>& l0,
                       std::vector<int>& l1, std::vector<int>& first) {
    const int nlp = (int)off.size() - 1;
    first.assign(nlp + 1, 0);
    for (int b = 0; b < nlp; ++b) {
        first[b] = (int)lp.size();
        long long a = off[b];
        if (off[b + 1] == off[b]) {  // an LP without lines still owns one empty tile
            lp.push_back(b);
            l0.push_back((int)a);
            l1.push_back((int)a);
            continue;
        }
        for (; a < off[b + 1]; a += per_tile) {
            lp.push_back(b);
            l0.push_back((int)a);
            l1.push_back((int)std::min<long long>(a + per_tile, off[b + 1]));
        }
    }
    first[nlp] = (int)lp.size();
}

int solve_batch(Ctx& ctx, const mc_lp* lps, int count, const mc_pdlp_options* o, const double* const* x0,
                const double* const* y0, double* const* x_out, double* const* y_out, mc_pdlp_result* results) {
    ctx.drop_session();  // the batch reuses the arena
    const double t_begin = now_ms();
    if (!lps || count <= 0 || !results) return set_error(MC_ERR_INVALID_ARGUMENT, "empty batch");
    TRY(validate_options(o));
    const bool mixed = o->precision == MC_PRECISION_FP32_REFINE;
    std::vector<long long> col_off(count + 1, 0), row_off(count + 1, 0), nnz_off(count + 1, 0);
    for (int b = 0; b < count; ++b) {
        std::memset(&results[b], 0, sizeof(mc_pdlp_result));
        TRY(validate_lp(&lps[b]));
        col_off[b + 1] = col_off[b] + lps[b].num_cols;
        row_off[b + 1] = row_off[b] + lps[b].num_rows;
        nnz_off[b + 1] = nnz_off[b] + lps[b].nnz;
    }
    const long long n = col_off[count], m = row_off[count], nnz = nnz_off[count];
    if (n >= (1LL << 31) - 1 || m >= (1LL << 31) - 1 || nnz >= (1LL << 31) - 1)
        return set_error(MC_ERR_RESOURCE_LIMIT, "packed batch beyond int32 indices");
    cudaStream_t s = ctx.stream;
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
        ctx.launches[q] = 0;
        ctx.kernel_ms[q] = 0.0;
    }
    ctx.profiling = o->profile_kernels != 0;
    ctx.pending.clear();
    ctx.prof_used = 0;
    ctx.release_graphs();

    // lanes per line from the packed means; tiles of one block-step (kBlock/G
    // lines): the LPs still running late in a batch are spread over as many
    // blocks as possible (measured on B200 on the 256-LP batch: 23% faster
    // than tiles of four block-steps)
    const int gc = valid_lanes(o->lanes_per_column) ? o->lanes_per_column : pick_lanes(n ? (double)nnz / n : 1.0);
    const int gr = valid_lanes(o->lanes_per_row) ? o->lanes_per_row : pick_lanes(m ? (double)nnz / m : 1.0);
    std::vector<int> ct_lp, ct_l0, ct_l1, ct_first, rt_lp, rt_l0, rt_l1, rt_first;
    make_tiles(col_off, kBlock / gc, ct_lp, ct_l0, ct_l1, ct_first);
    make_tiles(row_off, kBlock / gr, rt_lp, rt_l0, rt_l1, rt_first);
    const int nct = (int)ct_lp.size(), nrt = (int)rt_lp.size();
    if (nct > kMaxTiles || nrt > kMaxTiles)
        return set_error(MC_ERR_RESOURCE_LIMIT, "batch needs %d/%d tiles (limit %d)", nct, nrt, kMaxTiles);

    // ---- arena
    Layout L;
    const size_t o_cs = L.add<int>(n + 1), o_ri = L.add<int>(nnz + 16), o_cv = L.add<double>(nnz + 16);
    const size_t o_rs = L.add<int>(m + 1), o_ci = L.add<int>(nnz + 16), o_rv = L.add<double>(nnz + 16);
    const size_t o_cursor = L.add<int>(m), o_long = L.add<int>(m), o_counters = L.add<int>(4);
    const size_t o_scan = L.add<int>((m + 1) / kScanTile + 4096);
    const size_t o_tiles = L.add<int>(3LL * (nct + nrt) + 2LL * (count + 1));
    size_t o_n[12], o_m[10];
    for (auto& v : o_n) v = L.add<double>(n);
    for (auto& v : o_m) v = L.add<double>(m);
    const size_t o_part = L.add<double>((long long)NUM_SLOTS * kMaxTiles);
    const size_t o_st = L.add<DevState>(count + 1);
    const size_t o_off = L.add<double>(2LL * count);
    const size_t o_flags = L.add<int>(count);
    const size_t o_cert = L.add<int>(2LL * count);
    const size_t o_yprev = L.add<double>(m), o_dray = L.add<double>(m);
    bool any_warm = false;
    for (int b = 0; b < count; ++b)
        any_warm = any_warm || (x0 && x0[b] && lps[b].num_cols > 0) || (y0 && y0[b] && lps[b].num_rows > 0);
    const size_t o_warm = any_warm ? L.add<int>(count) : 0;
    const size_t o_warm_x = any_warm ? L.add<double>(n) : 0;
    const size_t o_warm_y = any_warm ? L.add<double>(m) : 0;
    const size_t o_active = L.add<int>(2LL * kMaxTiles + 2);
    const size_t o_lp_offset = L.add<int>(2LL * (count + 1));
    // (x-bar, dx) pairs of the step-size iterations, in the iterate type
    const size_t o_xdx = mixed ? L.add<float>(2LL * n) : L.add<double>(2LL * n);
    const bool tune = o->lanes_per_column == 0 || o->lanes_per_row == 0;
    size_t o_save_n[3] = {0, 0, 0}, o_save_m[2] = {0, 0};
    if (tune) {
        for (auto& v : o_save_n) v = L.add<double>(n);
        for (auto& v : o_save_m) v = L.add<double>(m);
    }
    // mixed form: FP32 matrix copies, FP32 correction iterates and cycle data
    size_t o_f_cscv = 0, o_f_csrv = 0, o_fn[8] = {}, o_fm[7] = {};
    if (mixed) {
        o_f_cscv = L.add<float>(nnz + 16);
        o_f_csrv = L.add<float>(nnz + 16);
        for (auto& v : o_fn) v = L.add<float>(n);
        for (auto& v : o_fm) v = L.add<float>(m);
    }
    // iterates: x, x_bar, x_avg, dx (columns); y, y_avg, ax_bar (rows)
    size_t o_it_n[4], o_it_m[3];
    for (auto& v : o_it_n) v = L.add<double>(n);
    for (auto& v : o_it_m) v = L.add<double>(m);
    TRY(ctx.arena.reserve(L.offset));
    char* A = static_cast<char*>(ctx.arena.base);
    auto at = [&](size_t off) { return static_cast<void*>(A + off); };
    int* cs = static_cast<int*>(at(o_cs));
    int* ri = static_cast<int*>(at(o_ri));
    double* cv = static_cast<double*>(at(o_cv));
    int* rs = static_cast<int*>(at(o_rs));
    int* ci = static_cast<int*>(at(o_ci));
    double* rv = static_cast<double*>(at(o_rv));
    double* obj_in = static_cast<double*>(at(o_n[0]));
    double* lo_in = static_cast<double*>(at(o_n[1]));
    double* hi_in = static_cast<double*>(at(o_n[2]));
    double* c = static_cast<double*>(at(o_n[3]));
    double* lo = static_cast<double*>(at(o_n[4]));
    double* hi = static_cast<double*>(at(o_n[5]));
    double* c_orig = static_cast<double*>(at(o_n[6]));
    double* lo_orig = static_cast<double*>(at(o_n[7]));
    double* hi_orig = static_cast<double*>(at(o_n[8]));
    double* col_norm = static_cast<double*>(at(o_n[9]));
    double* col_scale = static_cast<double*>(at(o_n[10]));
    double* rlo_in = static_cast<double*>(at(o_m[0]));
    double* rhi_in = static_cast<double*>(at(o_m[1]));
    double* blo = static_cast<double*>(at(o_m[2]));
    double* bhi = static_cast<double*>(at(o_m[3]));
    double* blo_orig = static_cast<double*>(at(o_m[4]));
    double* bhi_orig = static_cast<double*>(at(o_m[5]));
    double* row_norm = static_cast<double*>(at(o_m[6]));
    double* row_scale = static_cast<double*>(at(o_m[7]));
    double* partials = static_cast<double*>(at(o_part));
    DevState* st = static_cast<DevState*>(at(o_st));
    double* offsets = static_cast<double*>(at(o_off));
    double* signs = offsets + count;
    int* flags = static_cast<int*>(at(o_flags));
    int* cert_idx = static_cast<int*>(at(o_cert));
    double* x_work[4];
    for (int q = 0; q < 4; ++q) x_work[q] = static_cast<double*>(at(o_it_n[q]));
    double* y_work[3];
    for (int q = 0; q < 3; ++q) y_work[q] = static_cast<double*>(at(o_it_m[q]));
    double* stage_x = static_cast<double*>(at(o_n[11]));
    double* stage_y = static_cast<double*>(at(o_m[8]));

    // ---- uploads (cudaMemcpyDefault: host or device arrays), per-LP validation, index shift
    CU(cudaEventRecord(ctx.ev_a, s));
    int* counters = static_cast<int*>(at(o_counters));
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    for (int b = 0; b < count; ++b) {
        const mc_lp& lp = lps[b];
        const long long nb = lp.num_cols, mb = lp.num_rows, zb = lp.nnz;
        CU(cudaMemcpyAsync(cs + col_off[b], lp.col_start, sizeof(int) * (size_t)(nb + 1), cudaMemcpyDefault, s));
        if (zb) {
            CU(cudaMemcpyAsync(ri + nnz_off[b], lp.row_index, sizeof(int) * (size_t)zb, cudaMemcpyDefault, s));
            CU(cudaMemcpyAsync(cv + nnz_off[b], lp.value, sizeof(double) * (size_t)zb, cudaMemcpyDefault, s));
        }
        if (nb) {
            CU(cudaMemcpyAsync(obj_in + col_off[b], lp.objective, sizeof(double) * nb, cudaMemcpyDefault, s));
            CU(cudaMemcpyAsync(lo_in + col_off[b], lp.var_lower, sizeof(double) * nb, cudaMemcpyDefault, s));
            CU(cudaMemcpyAsync(hi_in + col_off[b], lp.var_upper, sizeof(double) * nb, cudaMemcpyDefault, s));
        }
        if (mb) {
            CU(cudaMemcpyAsync(rlo_in + row_off[b], lp.row_lower, sizeof(double) * mb, cudaMemcpyDefault, s));
            CU(cudaMemcpyAsync(rhi_in + row_off[b], lp.row_upper, sizeof(double) * mb, cudaMemcpyDefault, s));
        }
        if (nb > 0 && zb > 0) {  // validate in the LP's own numbering, then shift
            ctx.begin_launch(MC_KERNEL_SETUP);
            k_validate_csc<<<(int)((nb + kBlock - 1) / kBlock), kBlock, 0, s>>>(
                (int)mb, (int)nb, zb, cs + col_off[b], ri + nnz_off[b], cv + nnz_off[b], counters + 2);
            ctx.end_launch();
        }
        if (nb > 0) {
            ctx.begin_launch(MC_KERNEL_SETUP);
            kb_shift_indices<<<blocks_for(ctx, zb + nb, kBlock), kBlock, 0, s>>>(
                cs + col_off[b], ri + nnz_off[b], (int)nb, zb, (int)nnz_off[b], (int)row_off[b]);
            ctx.end_launch();
        }
    }
    {
        const int total = (int)nnz;
        CU(cudaMemcpyAsync(cs + n, &total, sizeof(int), cudaMemcpyHostToDevice, s));
    }
    // starting points: packed like the model, a flag per LP says which parts exist
    int* warm = any_warm ? static_cast<int*>(at(o_warm)) : nullptr;
    double* warm_x = any_warm ? static_cast<double*>(at(o_warm_x)) : nullptr;
    double* warm_y = any_warm ? static_cast<double*>(at(o_warm_y)) : nullptr;
    std::vector<int> warm_host(any_warm ? count : 0, 0);
    for (int b = 0; b < count && any_warm; ++b) {
        if (x0 && x0[b] && lps[b].num_cols > 0) {
            warm_host[b] |= 1;
            CU(cudaMemcpyAsync(warm_x + col_off[b], x0[b], sizeof(double) * lps[b].num_cols, cudaMemcpyDefault, s));
        }
        if (y0 && y0[b] && lps[b].num_rows > 0) {
            warm_host[b] |= 2;
            CU(cudaMemcpyAsync(warm_y + row_off[b], y0[b], sizeof(double) * lps[b].num_rows, cudaMemcpyDefault, s));
        }
    }
    if (any_warm) CU(cudaMemcpyAsync(warm, warm_host.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
    std::vector<double> host_off(2 * (size_t)count);
    for (int b = 0; b < count; ++b) {
        host_off[b] = lps[b].objective_offset;
        host_off[count + b] = lps[b].objective_sense == MC_MAXIMIZE ? -1.0 : 1.0;
    }
    CU(cudaMemcpyAsync(offsets, host_off.data(), sizeof(double) * host_off.size(), cudaMemcpyHostToDevice, s));
    // tile tables (lp, l0, l1 of every column tile and row tile, then each LP's
    // tile ranges), in one device buffer sized for the finest tiling
    std::vector<int> tiles_host;
    int* tiles = static_cast<int*>(at(o_tiles));
    auto upload_tiles = [&](int steps) -> int {
        ct_lp.clear(), ct_l0.clear(), ct_l1.clear(), rt_lp.clear(), rt_l0.clear(), rt_l1.clear();
        make_tiles(col_off, steps * (kBlock / gc), ct_lp, ct_l0, ct_l1, ct_first);
        make_tiles(row_off, steps * (kBlock / gr), rt_lp, rt_l0, rt_l1, rt_first);
        tiles_host.clear();
        for (auto* v : {&ct_lp, &ct_l0, &ct_l1, &rt_lp, &rt_l0, &rt_l1, &ct_first, &rt_first})
            tiles_host.insert(tiles_host.end(), v->begin(), v->end());
        CU(cudaMemcpyAsync(tiles, tiles_host.data(), sizeof(int) * tiles_host.size(), cudaMemcpyHostToDevice, s));
        return MC_OK;
    };
    TRY(upload_tiles(1));
    CU(cudaMemsetAsync(ri + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(cv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(ci + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(rv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(flags, 0, sizeof(int) * count, s));
    CU(cudaMemsetAsync(cert_idx, 0x7f, sizeof(int) * 2 * (size_t)count, s));  // "none" above any index
    CU(cudaMemsetAsync(at(o_dray), 0, sizeof(double) * (size_t)m, s));
    CU(cudaMemsetAsync(st, 0, sizeof(DevState) * (count + 1), s));
    CU(cudaEventRecord(ctx.ev_b, s));
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    if (bad) return set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix in the batch (flags %d)", bad);

    BatchRefs B;
    B.st = st;
    B.offset = offsets;
    B.flags = flags;
    B.cert_idx = cert_idx;
    B.y_prev = static_cast<double*>(at(o_yprev));
    B.dray = static_cast<double*>(at(o_dray));
    B.nlp = count;
    B.warm = warm;
    B.warm_x = warm_x;
    B.warm_y = warm_y;
    int* active = static_cast<int*>(at(o_active));
    B.active = active;
    B.active_count = active + 2LL * kMaxTiles;
    // point B's tables into the buffer as laid out for the current tiling
    auto bind_tiles = [&](BatchRefs& R) {
        const int c = (int)ct_lp.size(), r = (int)rt_lp.size();
        int* tp = tiles;
        R.cols.lp = tp; tp += c;
        R.cols.l0 = tp; tp += c;
        R.cols.l1 = tp; tp += c;
        R.rows.lp = tp; tp += r;
        R.rows.l0 = tp; tp += r;
        R.rows.l1 = tp; tp += r;
        R.cols.first = tp; tp += count + 1;
        R.rows.first = tp;
        R.cols.ntiles = c;
        R.rows.ntiles = r;
    };
    bind_tiles(B);

    // ---- setup: transpose, Ruiz per LP, data per LP
    TRY(build_csr(ctx, (int)m, (int)n, nnz, cs, ri, cv, rs, ci, rv, static_cast<int*>(at(o_cursor)),
                  static_cast<int*>(at(o_long)), counters, static_cast<int*>(at(o_scan))));
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_fill<double><<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(row_scale, m, 1.0);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_fill<double><<<blocks_for(ctx, n, kBlock), kBlock, 0, s>>>(col_scale, n, 1.0);
    ctx.end_launch();
    double* r_tmp = y_work[2];
    double* c_tmp = x_work[3];
    const long long passes = o->ruiz_scaling ? o->ruiz_iterations : 0;
    for (long long pass = 0; pass < passes && nnz > 0; ++pass) {
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_line_max<<<nct, kBlock, 0, s>>>(cs, cv, c_tmp, partials, SLOT_A, B.cols, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_line_max<<<nrt, kBlock, 0, s>>>(rs, rv, r_tmp, partials, SLOT_B, B.rows, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_check<<<count, 256, 0, s>>>(partials, B, 1e-3);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_deltas<<<nrt, kBlock, 0, s>>>(r_tmp, row_scale, B.rows, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_deltas<<<nct, kBlock, 0, s>>>(c_tmp, col_scale, B.cols, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_rescale<<<nct, kBlock, 0, s>>>(cs, ri, cv, c_tmp, r_tmp, B.cols, st);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kb_ruiz_rescale<<<nrt, kBlock, 0, s>>>(rs, ci, rv, r_tmp, c_tmp, B.rows, st);
        ctx.end_launch();
    }
    Iterates<double> P;
    P.m = (int)m;
    P.n = (int)n;
    P.csc_start = cs;
    P.csc_row = ri;
    P.csc_val = cv;
    P.csr_start = rs;
    P.csr_col = ci;
    P.csr_val = rv;
    P.c = c;
    P.lo = lo;
    P.hi = hi;
    P.blo = blo;
    P.bhi = bhi;
    P.col_norm = col_norm;
    P.row_norm = row_norm;
    P.x = x_work[0];
    P.x_bar = x_work[1];
    P.x_avg = x_work[2];
    P.dx = x_work[3];
    P.xdx = mixed ? nullptr : static_cast<double*>(at(o_xdx));
    P.y = y_work[0];
    P.y_avg = y_work[1];
    P.ax_bar = y_work[2];
    P.partials = partials;
    P.st = st;
    Original O{c_orig, obj_in, lo_orig, hi_orig, blo_orig, bhi_orig, col_scale, row_scale, 0.0};
    ctx.begin_launch(MC_KERNEL_SETUP);
    kb_setup_cols<<<nct, kBlock, 0, s>>>(cs, cv, obj_in, lo_in, hi_in, col_scale, signs, P, O, partials, B);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    kb_setup_rows<<<nrt, kBlock, 0, s>>>(rs, ci, rv, rlo_in, rhi_in, row_scale, col_scale, lo_in, hi_in, P, O,
                                         partials, B);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    kb_setup_scalars<<<count, 256, 0, s>>>(partials, B, o->initial_primal_weight, o->step_size_reduction);
    ctx.end_launch();
    TRY(ctx.launch_check("batch setup"));

    Controls ctl{o->primal_tolerance, o->dual_tolerance, o->gap_tolerance, o->restart_reduction_factor,
                 o->primal_weight_smoothing, o->restart_every, o->restart_strategy, o->adaptive_step_size,
                 o->adaptive_primal_weight};
    TraceBuf tr{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const int poll_every = o->check_every_chunks > 0 ? o->check_every_chunks : 1;
    auto setup_common = [&](BatchCommon& e) {
        e.B = B;
        e.global = st + count;
        e.g_col = gc;
        e.g_row = gr;
        e.active = active;
        e.active_count = active + 2LL * kMaxTiles;
        e.lp_offset = static_cast<int*>(at(o_lp_offset));
    };
    // lanes: the autotuner where the options leave them open, else as given
    auto tune_if_asked = [&](auto& e) -> int {
        if (!tune) return MC_OK;
        void* save_n[3];
        void* save_m[2];
        for (int q = 0; q < 3; ++q) save_n[q] = at(o_save_n[q]);
        for (int q = 0; q < 2; ++q) save_m[q] = at(o_save_m[q]);
        const int keep_col = e.g_col, keep_row = e.g_row;
        // the block shape: tiles of `steps` block-steps, re-bound and re-queued
        auto retile = [&](int steps) -> int {
            TRY(upload_tiles(steps));
            bind_tiles(e.B);
            return e.compact(ctx);
        };
        TRY(tune_lanes(ctx, e, o->precision, save_n, save_m, retile));
        if (valid_lanes(o->lanes_per_column)) e.g_col = keep_col;
        if (valid_lanes(o->lanes_per_row)) e.g_row = keep_row;
        B = e.B;  // the tables the solve ran with (for the output stage)
        return MC_OK;
    };
    float* f_xa = nullptr;
    float* f_ya = nullptr;
    if (!mixed) {
        EngineBatch eng;
        setup_common(eng);
        eng.P = P;
        eng.O = O;
        TRY(eng.compact(ctx));
        TRY(tune_if_asked(eng));
        TRY(run_chunks(ctx, eng, eng.global, o->max_iterations, o->restart_every, poll_every, ctl, tr));
    } else {
        EngineBatchMixed eng;
        setup_common(eng);
        float* f_cscv = static_cast<float*>(at(o_f_cscv));
        float* f_csrv = static_cast<float*>(at(o_f_csrv));
        float* fn[8];
        float* fm[7];
        for (int q = 0; q < 8; ++q) fn[q] = static_cast<float*>(at(o_fn[q]));
        for (int q = 0; q < 7; ++q) fm[q] = static_cast<float*>(at(o_fm[q]));
        const int nbz = blocks_for(ctx, nnz + 16, kBlock) * 4;
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, cv, f_cscv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, rv, f_csrv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<blocks_for(ctx, n, kBlock), kBlock, 0, s>>>(n, col_norm, fn[3]);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(m, row_norm, fm[0]);
        ctx.end_launch();
        Iterates<float>& F = eng.P;
        F.m = (int)m;
        F.n = (int)n;
        F.csc_start = cs;
        F.csc_row = ri;
        F.csc_val = f_cscv;
        F.csr_start = rs;
        F.csr_col = ci;
        F.csr_val = f_csrv;
        F.c = fn[0];
        F.lo = fn[1];
        F.hi = fn[2];
        F.blo = nullptr;  // the mixed dual step reads r_lo / r_hi instead
        F.bhi = nullptr;
        F.col_norm = fn[3];
        F.row_norm = fm[0];
        F.x = fn[4];
        F.x_bar = fn[5];
        F.x_avg = fn[6];
        F.dx = fn[7];
        F.xdx = static_cast<float*>(at(o_xdx));
        F.y = fm[1];
        F.y_avg = fm[2];
        F.ax_bar = fm[3];
        F.partials = partials;
        F.st = st;
        MixedState& M = eng.M;
        M.x_hat = P.x;  // every LP's FP64 start point is its first base
        M.y_hat = P.y;
        M.ax_full = P.ax_bar;
        M.aty_full = P.dx;
        M.c64 = c;
        M.lo64 = lo;
        M.hi64 = hi;
        M.blo64 = blo;
        M.bhi64 = bhi;
        M.csc_val64 = cv;
        M.csr_val64 = rv;
        M.g = fn[0];
        M.lo = fn[1];
        M.hi = fn[2];
        M.r_lo = fm[4];
        M.r_hi = fm[5];
        M.yb = fm[6];
        eng.O = O;
        f_xa = F.x_avg;
        f_ya = F.y_avg;
        for (int q = 4; q < 8; ++q) CU(cudaMemsetAsync(fn[q], 0, sizeof(float) * (size_t)n, s));
        for (int q = 1; q < 4; ++q) CU(cudaMemsetAsync(fm[q], 0, sizeof(float) * (size_t)m, s));
        TRY(eng.compact(ctx));
        // the first correction LP of every running LP, around its start point
        TRY(eng.residual_pass(ctx));
        TRY(eng.recenter(ctx, 1));
        TRY(tune_if_asked(eng));
        TRY(run_chunks(ctx, eng, eng.global, o->max_iterations, o->restart_every, poll_every, ctl, tr));
    }
    CU(cudaEventRecord(ctx.ev_c, s));

    // ---- outputs
    ctx.begin_launch(MC_KERNEL_OTHER);
    kb_unscale_out<<<B.cols.ntiles + B.rows.ntiles, kBlock, 0, s>>>(mixed ? P.x : P.x_avg, f_xa, mixed ? P.y : P.y_avg, f_ya, col_scale,
                                                row_scale, stage_x, stage_y, B);
    ctx.end_launch();
    TRY(ctx.launch_check("batch unscale"));
    for (int b = 0; b < count; ++b) {
        if (x_out && x_out[b] && lps[b].num_cols > 0)
            CU(cudaMemcpyAsync(x_out[b], stage_x + col_off[b], sizeof(double) * lps[b].num_cols, cudaMemcpyDefault, s));
        if (y_out && y_out[b] && lps[b].num_rows > 0)
            CU(cudaMemcpyAsync(y_out[b], stage_y + row_off[b], sizeof(double) * lps[b].num_rows, cudaMemcpyDefault, s));
    }
    std::vector<DevState> hs(count);
    CU(cudaMemcpyAsync(hs.data(), st, sizeof(DevState) * count, cudaMemcpyDeviceToHost, s));
    std::vector<int> hcert(2 * (size_t)count);
    CU(cudaMemcpyAsync(hcert.data(), cert_idx, sizeof(int) * hcert.size(), cudaMemcpyDeviceToHost, s));
    CU(cudaEventRecord(ctx.ev_d, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    float h2d = 0.f, kern = 0.f, d2h = 0.f;
    CU(cudaEventElapsedTime(&h2d, ctx.ev_a, ctx.ev_b));
    CU(cudaEventElapsedTime(&kern, ctx.ev_b, ctx.ev_c));
    CU(cudaEventElapsedTime(&d2h, ctx.ev_c, ctx.ev_d));
    long long total = 0;
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) total += ctx.launches[q];
    const double total_ms = now_ms() - t_begin;
    for (int b = 0; b < count; ++b) {
        mc_pdlp_result& r = results[b];
        std::snprintf(r.backend_actually_used, sizeof r.backend_actually_used, "cuda");
        r.tolerance = o->primal_tolerance;
        r.certificate_index = -1;
        if (lps[b].num_rows == 0 || lps[b].num_cols == 0) {
            r.status = MC_PDLP_OPTIMAL;
            fill_message(&r, "trivial");
            continue;
        }
        const DevState& S = hs[b];
        r.status = S.status;
        r.objective = S.objective;
        r.primal_infeasibility = S.primal_infeas;
        r.dual_infeasibility = S.dual_infeas;
        r.duality_gap = S.gap;
        r.iterations = S.iter;
        r.certificate = S.status == MC_PDLP_INFEASIBLE_OR_UNBOUNDED ? S.cert : MC_CERT_NONE;
        r.certificate_index = r.certificate == MC_CERT_CROSSED_BOUNDS ? hcert[b]
                              : r.certificate == MC_CERT_ROW_ACTIVITY ? hcert[count + b]
                                                                      : -1;
        fill_message(&r, S.status == MC_PDLP_OPTIMAL ? "PDLP converged"
                         : r.certificate == MC_CERT_CROSSED_BOUNDS ? "infeasible: crossed variable bounds"
                         : r.certificate == MC_CERT_ROW_ACTIVITY ? "infeasible: row activity outside its bounds"
                         : r.certificate == MC_CERT_DUAL_RAY ? "infeasible: dual ray (Farkas certificate in dual)"
                         : S.status == MC_PDLP_NUMERICAL_FAILURE ? "non-finite iterate or residual"
                                                                 : "iteration limit reached");
        r.h2d_ms = h2d;
        r.kernel_ms = kern;
        r.d2h_ms = d2h;
        r.total_ms = total_ms;
        r.ruiz_iterations_executed = o->ruiz_scaling ? S.ruiz_passes : 0;
        r.restarts = S.restarts;
        r.final_primal_weight = S.omega;
        r.final_step_size = S.eta;
        r.kernel_launches = total;
        r.refinement_rounds = mixed ? S.restarts : 0;  // each restart re-centres the LP's FP64 base
        r.inner_iterations = mixed ? S.iter : 0;
        for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
            r.launches_by_kind[q] = ctx.launches[q];
            r.kernel_ms_by_kind[q] = ctx.kernel_ms[q];
        }
    }
    return MC_OK;
}

}  // namespace mc
