// Host driver of the batched solve (included once, by engine.cu after solve.cuh).
#pragma once

#include "batch_kernels.cuh"
#include "solve.cuh"

#include <vector>

namespace mc {

struct EngineBatch {
    Iterates<double> P;
    Original O;
    BatchRefs B;
    DevState* global = nullptr;  // poll flag: every LP done
    int g_col = 1, g_row = 1;

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        const int nc = B.cols.ntiles, nr = B.rows.ntiles;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) {
            MC_DISPATCH_G(g_col, (kb_primal<G, true><<<nc, kBlock, 0, s>>>(P, B, k)));
        } else {
            MC_DISPATCH_G(g_col, (kb_primal<G, false><<<nc, kBlock, 0, s>>>(P, B, k)));
        }
        ctx.end_launch();
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            MC_DISPATCH_G(g_row, (kb_dual_probe<G><<<nr, kBlock, 0, s>>>(P, B)));
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            kb_step_size<<<B.nlp, 256, 0, s>>>(P.partials, B, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kb_dual_apply<<<nr, kBlock, 0, s>>>(P, B, k);
            ctx.end_launch();
        } else {
            ctx.begin_launch(MC_KERNEL_DUAL);
            MC_DISPATCH_G(g_row, (kb_dual<G><<<nr, kBlock, 0, s>>>(P, B, k)));
            ctx.end_launch();
        }
        return ctx.launch_check("batch iteration");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf&) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_row, (kb_residual_rows<G><<<B.rows.ntiles, kBlock, 0, s>>>(P, O, B)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        MC_DISPATCH_G(g_col, (kb_residual_cols<G><<<B.cols.ntiles, kBlock, 0, s>>>(P, O, B)));
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kb_finalize<<<B.nlp, 256, 0, s>>>(P.partials, B, span, final_pass, ctl);
        ctx.end_launch();
        if (!final_pass) {
            ctx.begin_launch(MC_KERNEL_OTHER);
            kb_restart_copy<<<B.cols.ntiles + B.rows.ntiles, kBlock, 0, s>>>(P, B);
            ctx.end_launch();
        }
        ctx.begin_launch(MC_KERNEL_OTHER);
        kb_all_done<<<1, 256, 0, s>>>(B.st, B.nlp, global);
        ctx.end_launch();
        return ctx.launch_check("batch check");
    }
};

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

int solve_batch(Ctx& ctx, const mc_lp* lps, int count, const mc_pdlp_options* o, double* const* x_out,
                double* const* y_out, mc_pdlp_result* results) {
    const double t_begin = now_ms();
    if (!lps || count <= 0 || !results) return set_error(MC_ERR_INVALID_ARGUMENT, "empty batch");
    TRY(validate_options(o));
    if (o->precision != MC_PRECISION_FP64)
        return set_error(MC_ERR_INVALID_ARGUMENT, "batched solves run the FP64 form");
    if (o->lanes_per_column == -1 || o->lanes_per_row == -1)
        return set_error(MC_ERR_INVALID_ARGUMENT, "batched solves use the lane kernels");
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

    // lanes per line from the packed means, tiles of four block-steps
    const int gc = valid_lanes(o->lanes_per_column) ? o->lanes_per_column : pick_lanes(n ? (double)nnz / n : 1.0);
    const int gr = valid_lanes(o->lanes_per_row) ? o->lanes_per_row : pick_lanes(m ? (double)nnz / m : 1.0);
    std::vector<int> ct_lp, ct_l0, ct_l1, ct_first, rt_lp, rt_l0, rt_l1, rt_first;
    make_tiles(col_off, 4 * kBlock / gc, ct_lp, ct_l0, ct_l1, ct_first);
    make_tiles(row_off, 4 * kBlock / gr, rt_lp, rt_l0, rt_l1, rt_first);
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
    std::vector<double> host_off(2 * (size_t)count);
    for (int b = 0; b < count; ++b) {
        host_off[b] = lps[b].objective_offset;
        host_off[count + b] = lps[b].objective_sense == MC_MAXIMIZE ? -1.0 : 1.0;
    }
    CU(cudaMemcpyAsync(offsets, host_off.data(), sizeof(double) * host_off.size(), cudaMemcpyHostToDevice, s));
    std::vector<int> tiles_host;
    tiles_host.reserve(3 * (nct + nrt) + 2 * (count + 1));
    for (auto* v : {&ct_lp, &ct_l0, &ct_l1, &rt_lp, &rt_l0, &rt_l1, &ct_first, &rt_first})
        tiles_host.insert(tiles_host.end(), v->begin(), v->end());
    int* tiles = static_cast<int*>(at(o_tiles));
    CU(cudaMemcpyAsync(tiles, tiles_host.data(), sizeof(int) * tiles_host.size(), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(ri + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(cv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(ci + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(rv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(flags, 0, sizeof(int) * count, s));
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
    B.nlp = count;
    int* tp = tiles;
    B.cols.lp = tp; tp += nct;
    B.cols.l0 = tp; tp += nct;
    B.cols.l1 = tp; tp += nct;
    B.rows.lp = tp; tp += nrt;
    B.rows.l0 = tp; tp += nrt;
    B.rows.l1 = tp; tp += nrt;
    B.cols.first = tp; tp += count + 1;
    B.rows.first = tp;
    B.cols.ntiles = nct;
    B.rows.ntiles = nrt;

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

    EngineBatch eng;
    eng.P = P;
    eng.O = O;
    eng.B = B;
    eng.global = st + count;
    eng.g_col = gc;
    eng.g_row = gr;
    Controls ctl{o->primal_tolerance, o->dual_tolerance, o->gap_tolerance, o->restart_reduction_factor,
                 o->primal_weight_smoothing, o->restart_every, o->restart_strategy, o->adaptive_step_size,
                 o->adaptive_primal_weight};
    TraceBuf tr{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    ctx.begin_launch(MC_KERNEL_OTHER);
    kb_all_done<<<1, 256, 0, s>>>(st, count, eng.global);
    ctx.end_launch();
    const int poll_every = o->check_every_chunks > 0 ? o->check_every_chunks : 1;
    TRY(run_chunks(ctx, eng, eng.global, o->max_iterations, o->restart_every, poll_every, ctl, tr));
    CU(cudaEventRecord(ctx.ev_c, s));

    // ---- outputs
    ctx.begin_launch(MC_KERNEL_OTHER);
    kb_unscale_out<<<nct + nrt, kBlock, 0, s>>>(P, col_scale, row_scale, stage_x, stage_y, B);
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
        fill_message(&r, S.status == MC_PDLP_OPTIMAL ? "PDLP converged"
                         : S.status == MC_PDLP_INFEASIBLE_OR_UNBOUNDED ? "infeasible: certified at setup"
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
        for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
            r.launches_by_kind[q] = ctx.launches[q];
            r.kernel_ms_by_kind[q] = ctx.kernel_ms[q];
        }
    }
    return MC_OK;
}

}  // namespace mc
