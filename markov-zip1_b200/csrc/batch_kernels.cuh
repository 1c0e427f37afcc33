// Batched PDLP: many independent LPs of uneven size solved together.
//
// The LPs are packed block-diagonally into one CSC and one CSR (column block
// b holds LP b's columns, row block b its rows).  A tile is a run of
// consecutive lines (columns or rows) of ONE LP, so a block working on it
// reads that LP's scalars once (its DevState: eta, omega, averaging count,
// restart and termination state) and writes the tile's reduction partial to
// the tile's own slot.  The per-LP reductions then read the LP's tile range in
// order: every LP follows the reference algorithm
// (src/lp/first_order/pdlp.cpp:139-276) on its own -- own step size, own
// primal weight, own restarts and termination -- exactly as if it were solved
// alone, and the results are run-to-run deterministic.
//
// Work queue: the iteration kernels are persistent (one wave of resident
// blocks) and walk a compacted list of the tiles whose LP is still running,
// block b taking entries b, b + grid, b + 2 grid, ...  kb_compact and
// kb_fill_active rebuild the list after every restart check (the only place an
// LP terminates), so an LP that has converged costs nothing from its next
// chunk on, and the long tail where a few slow LPs run on alone costs only
// their own tiles.
//
// The row and column work inside a tile is the single-LP kernels' (lanes per
// line, cache policies, fused updates), so the per-nonzero cost is the same.
#pragma once

#include "common.cuh"
#include "iter_kernels.cuh"
#include "mixed.cuh"
#include "setup_kernels.cuh"

namespace mc {

struct TileTable {
    const int* lp;     // [ntiles] owning LP
    const int* l0;     // [ntiles] first line
    const int* l1;     // [ntiles] one past the last line
    const int* first;  // [nlp + 1] tile range of each LP
    int ntiles;
};

constexpr int kMaxTiles = 1 << 18;  // per-slot capacity of the batch partials buffer

struct BatchRefs {
    DevState* st;              // [nlp]
    const double* offset;      // [nlp] objective offsets
    int* flags;                // [nlp] setup certificates: 1 crossed bounds, 2 row activity
    int* cert_idx;             // [2 nlp] lowest crossed column, lowest failing row of each LP
                               // (LP-local indices; INT_MAX if none)
    double* y_prev;            // [m] dual average at the previous check (scaled; the start at setup)
    double* dray;              // [m] the ray candidate of the current check (scaled)
    const int* warm;           // [nlp] starting point given: 1 primal, 2 dual (NULL: none)
    const double* warm_x;      // [n] packed starting primal (original space)
    const double* warm_y;      // [m] packed starting dual
    TileTable cols, rows;
    const int* active;         // [2 * kMaxTiles] running column tiles, then running row tiles
    const int* active_count;   // [2] lengths of the two lists
    int nlp;
};

// The running tiles of one kind (0 columns, 1 rows), grid-strided over the
// persistent blocks; T is the tile's index in its table.
#define MC_FOR_ACTIVE(B, WHICH, T)                                                                  \
    for (int q_ = blockIdx.x, nq_ = B.active_count[WHICH]; q_ < nq_; q_ += gridDim.x)             \
        if (const int T = B.active[(WHICH) * kMaxTiles + q_]; true)

// Lines of tile T, G lanes per line; every thread of the block makes the same
// number of trips (the shuffles need all lanes).
#define MC_TILE_LINES(TT, T, LINE, VALID, SUB)                                                       \
    const int SUB = threadIdx.x % G;                                                                \
    const int tl1_ = TT.l1[T];                                                                      \
    for (int base_ = TT.l0[T], LINE = 0;                                                            \
         base_ < tl1_ && ((LINE = base_ + (int)(threadIdx.x / G)), true); base_ += kBlock / G)     \
        if (const bool VALID = LINE < tl1_; true)

// The Farkas test, evaluated in the residual pass on a dual ray candidate d:
// the change of the dual average since the previous check (unscaled), with
// its components on one-sided rows projected to the sign the finite bound
// allows (and zeroed on free rows).  For a primal infeasible LP the dual
// iterates diverge along a ray, so these differences point along it while
// the bounded part of the average cancels.  With g = A^T d,
//     L = sum_j (g_j > 0 ? g_j lo_j : g_j hi_j) <= g.x = d.(A x) <= U,
//     U = sum_i (d_i > 0 ? d_i hi_i : d_i lo_i)
// would hold for any x in the variable box that met the rows, so L > U proves
// the LP infeasible.  A nonzero g_j meeting an infinite bound makes L = -inf
// and is counted instead.  The scales bound the rounding of both sums (|bound|
// times sum |a d| per column, |d bound| per row), so a margin of 1e-9 of them
// cannot come from rounding.
struct RayTerms {
    double l = 0.0, cscale = 0.0, cinf = 0.0, u = 0.0, rscale = 0.0, rinf = 0.0;
    // the candidate of row i (scaled units) from the current and the previous
    // check's dual averages; the current one becomes the previous
    __device__ __forceinline__ static double candidate(const Original& O, int i, double y_now, double* y_prev) {
        double d = y_now - *y_prev;
        *y_prev = y_now;
        const double lo = O.blo[i], hi = O.bhi[i];
        const bool lo_inf = lo <= -1e299, hi_inf = hi >= 1e299;
        if (lo_inf && hi_inf) d = 0.0;
        else if (lo_inf) d = maxv(d, 0.0);
        else if (hi_inf) d = minv(d, 0.0);
        return d;
    }
    __device__ __forceinline__ void add_col(const Original& O, int j, double s, double s_abs) {
        add_col_b(O, j, s, s_abs, O.lo[j], O.hi[j]);
    }
    __device__ __forceinline__ void add_col_b(const Original& O, int j, double s, double s_abs, double lo,
                                              double hi) {
        const double g = __ddiv_rn(s, O.col_scale[j]);
        const double gabs = s_abs / O.col_scale[j];
        if (g != 0.0) {
            const double bnd = (g > 0.0) ? lo : hi;
            if (fabs(bnd) >= 1e299) {
                cinf += 1.0;
            } else {
                l += __dmul_rn(g, bnd);
                cscale += gabs * fabs(bnd);
            }
        }
    }
    __device__ __forceinline__ void add_row(const Original& O, int i, double d_scaled) {
        const double du = __dmul_rn(d_scaled, O.row_scale[i]);
        if (du == 0.0) return;
        const double bnd = (du > 0.0) ? O.bhi[i] : O.blo[i];
        if (fabs(bnd) >= 1e299) {
            rinf += 1.0;
        } else {
            const double t = __dmul_rn(du, bnd);
            u += t;
            rscale += fabs(t);
        }
    }
    __device__ __forceinline__ void store_cols(double* partials, double* scratch, int t) {
        l = block_reduce(l, scratch, OpSum());
        cscale = block_reduce(cscale, scratch, OpSum());
        cinf = block_reduce(cinf, scratch, OpSum());
        if (threadIdx.x == 0) {
            partials[SLOT_RAY_L * kMaxTiles + t] = l;
            partials[SLOT_RAY_CSCALE * kMaxTiles + t] = cscale;
            partials[SLOT_RAY_CINF * kMaxTiles + t] = cinf;
        }
    }
    __device__ __forceinline__ void store_rows(double* partials, double* scratch, int t) {
        u = block_reduce(u, scratch, OpSum());
        rscale = block_reduce(rscale, scratch, OpSum());
        rinf = block_reduce(rinf, scratch, OpSum());
        if (threadIdx.x == 0) {
            partials[SLOT_RAY_U * kMaxTiles + t] = u;
            partials[SLOT_RAY_RSCALE * kMaxTiles + t] = rscale;
            partials[SLOT_RAY_RINF * kMaxTiles + t] = rinf;
        }
    }
};

// ------------------------------------------------------------------ primal
template <int G, bool STEP, class T>
__global__ void __launch_bounds__(kBlock) kb_primal(Iterates<T> P, BatchRefs B, int k) {
    __shared__ double scratch[32];
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 0, t) {
        const DevState* st = B.st + B.cols.lp[t];
        const T step = T(st->eta / st->omega);
        const T cnt = T((double)(st->avg_count + k + 1));
        double acc = 0.0;
        MC_TILE_LINES(B.cols, t, j, valid, sub) {
            const bool owner = valid && sub == 0;
            T cn = T(1), cj = T(0), xo = T(0), lj = T(0), hj = T(0), xa = T(0);
            if (owner) {
                cn = ld_stream(P.col_norm + j);
                cj = ld_stream(P.c + j);
                xo = ld_stream(P.x + j);
                lj = ld_stream(P.lo + j);
                hj = ld_stream(P.hi + j);
                xa = ld_stream(P.x_avg + j);
            }
            const T aty = line_dot<G>(P.csc_start, P.csc_row, P.csc_val, P.y, j, valid, sub, pol);
            if (owner) {
                const T g = add_rn(cj, aty);
                const T tau = div_rn(step, cn);
                const T xp = clampv(sub_rn(xo, mul_rn(tau, g)), lj, hj);
                const T d = sub_rn(xp, xo);
                const T xb = sub_rn(mul_rn(T(2), xp), xo);
                if (STEP) {
                    st_keep2(P.xdx + 2LL * j, xb, d, pol);
                    acc += __dmul_rn(__dmul_rn((double)cn, (double)d), (double)d);
                } else {
                    st_keep(P.x_bar + j, xb, pol);
                }
                st_stream(P.x + j, xp);
                st_stream(P.x_avg + j, add_rn(xa, div_rn(sub_rn(xp, xa), cnt)));
            }
        }
        if (STEP) {
            acc = block_reduce(acc, scratch, OpSum());
            if (threadIdx.x == 0) P.partials[SLOT_DX * kMaxTiles + t] = acc;
        }
    }
}

// -------------------------------------------------------------------- dual
template <int G>
__global__ void __launch_bounds__(kBlock) kb_dual(Iterates<double> P, BatchRefs B, int k) {
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 1, t) {
        const DevState* st = B.st + B.rows.lp[t];
        const double sg = st->eta * st->omega;
        const double cnt = (double)(st->avg_count + k + 1);
        MC_TILE_LINES(B.rows, t, i, valid, sub) {
            RowData<double> r{};
            if (valid && sub == 0) r = load_row(P, i);
            const double ax = line_dot<G>(P.csr_start, P.csr_col, P.csr_val, P.x_bar, i, valid, sub, pol);
            if (valid && sub == 0) dual_update(P, i, r, ax, sg, cnt, pol);
        }
    }
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) kb_dual_probe(Iterates<T> P, BatchRefs B) {
    __shared__ double scratch[32];
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 1, t) {
        double acc = 0.0;
        MC_TILE_LINES(B.rows, t, i, valid, sub) {
            T axb, adx;
            line_dot2<G>(P.csr_start, P.csr_col, P.csr_val, P.xdx, i, valid, sub, axb, adx, pol);
            if (valid && sub == 0) {
                P.ax_bar[i] = axb;
                const double a = (double)adx;
                acc += __ddiv_rn(__dmul_rn(a, a), (double)P.row_norm[i]);
            }
        }
        acc = block_reduce(acc, scratch, OpSum());
        if (threadIdx.x == 0) P.partials[SLOT_ADX * kMaxTiles + t] = acc;
    }
}

// one block per LP: the adaptive eta rule (pdlp.cpp:207-219) on the LP's sums
__global__ void kb_step_size(const double* __restrict__ partials, BatchRefs B, Controls ctl) {
    __shared__ double scratch[32];
    const int lp = blockIdx.x;
    DevState* st = B.st + lp;
    if (st->done) return;
    const int c0 = B.cols.first[lp], c1 = B.cols.first[lp + 1];
    const int r0 = B.rows.first[lp], r1 = B.rows.first[lp + 1];
    const double dxn = reduce_partials(partials + SLOT_DX * kMaxTiles + c0, c1 - c0, scratch, OpSum());
    const double adx = reduce_partials(partials + SLOT_ADX * kMaxTiles + r0, r1 - r0, scratch, OpSum());
    if (threadIdx.x == 0 && ctl.adaptive_step && dxn > 1e-14 && adx > 1e-14) {
        const double L = sqrt(adx / dxn);
        if (L > 1e-6) {
            const double target = 0.95 / L;
            const double eta = st->eta;
            if (target < eta) st->eta = maxv(0.1, maxv(target, eta * 0.8));
            else if (target > 1.05 * eta && eta < 0.99) st->eta = minv(0.99, eta * 1.05);
        }
    }
}

__global__ void __launch_bounds__(kBlock) kb_dual_apply(Iterates<double> P, BatchRefs B, int k) {
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 1, t) {
        const DevState* st = B.st + B.rows.lp[t];
        const double sg = st->eta * st->omega;
        const double cnt = (double)(st->avg_count + k + 1);
        for (int i = B.rows.l0[t] + threadIdx.x; i < B.rows.l1[t]; i += blockDim.x)
            dual_update(P, i, P.ax_bar[i], sg, cnt, pol);
    }
}

// --------------------------------------------------------------- residuals
template <int G>
__global__ void __launch_bounds__(kBlock) kb_residual_rows(Iterates<double> P, Original O, BatchRefs B) {
    __shared__ double scratch[32];
    MC_FOR_ACTIVE(B, 1, t) {
        RowTerms acc;
        RayTerms ray;
        MC_TILE_LINES(B.rows, t, i, valid, sub) {
            double s = 0.0;
            if (valid) {
                const int b = P.csr_start[i], e = P.csr_start[i + 1];
                for (int p = b + sub; p < e; p += G) s = fma(P.csr_val[p], P.x_avg[P.csr_col[p]], s);
            }
            s = group_sum<G>(s);
            if (valid && sub == 0) {
                acc.add(O, i, s, P.y_avg[i]);
                const double d = RayTerms::candidate(O, i, P.y_avg[i], B.y_prev + i);
                B.dray[i] = d;
                ray.add_row(O, i, d);
            }
        }
        acc.vmax = block_reduce(acc.vmax, scratch, OpMax());
        acc.dsum = block_reduce(acc.dsum, scratch, OpSum());
        acc.bad = block_reduce(acc.bad, scratch, OpSum());
        if (threadIdx.x == 0) {
            P.partials[SLOT_ROW_MAX * kMaxTiles + t] = acc.vmax;
            P.partials[SLOT_ROW_DOBJ * kMaxTiles + t] = acc.dsum;
            P.partials[SLOT_NAN * kMaxTiles + t] = acc.bad;
        }
        ray.store_rows(P.partials, scratch, t);
    }
}

template <int G>
__global__ void __launch_bounds__(kBlock) kb_residual_cols(Iterates<double> P, Original O, BatchRefs B) {
    __shared__ double scratch[32];
    MC_FOR_ACTIVE(B, 0, t) {
        ColTerms acc;
        RayTerms ray;
        MC_TILE_LINES(B.cols, t, j, valid, sub) {
            double s = 0.0, sd = 0.0, sa = 0.0;
            if (valid) {
                const int b = P.csc_start[j], e = P.csc_start[j + 1];
                for (int p = b + sub; p < e; p += G) {
                    const int ii = P.csc_row[p];
                    const double a = P.csc_val[p], dv = B.dray[ii];
                    s = fma(a, P.y_avg[ii], s);
                    sd = fma(a, dv, sd);
                    sa = fma(fabs(a), fabs(dv), sa);
                }
            }
            s = group_sum<G>(s);
            sd = group_sum<G>(sd);
            sa = group_sum<G>(sa);
            if (valid && sub == 0) {
                acc.add(O, j, s, P.x_avg[j]);
                ray.add_col(O, j, sd, sa);
            }
        }
        acc.vmax = block_reduce(acc.vmax, scratch, OpMax());
        acc.dres = block_reduce(acc.dres, scratch, OpSum());
        acc.pobj = block_reduce(acc.pobj, scratch, OpSum());
        acc.dobj = block_reduce(acc.dobj, scratch, OpSum());
        acc.bad = block_reduce(acc.bad, scratch, OpSum());
        if (threadIdx.x == 0) {
            P.partials[SLOT_COL_MAX * kMaxTiles + t] = acc.vmax;
            P.partials[SLOT_COL_DRES * kMaxTiles + t] = acc.dres;
            P.partials[SLOT_COL_POBJ * kMaxTiles + t] = acc.pobj;
            P.partials[SLOT_COL_DOBJ * kMaxTiles + t] = acc.dobj;
            P.partials[SLOT_B * kMaxTiles + t] = acc.bad;
        }
        ray.store_cols(P.partials, scratch, t);
    }
}

// One block per LP: KKT scalars, termination, restart and primal weight of
// that LP (pdlp.cpp:229-261), as k_finalize for a single LP.
__global__ void kb_finalize(const double* __restrict__ partials, BatchRefs B, long long span, int final_pass,
                            Controls ctl) {
    __shared__ double scratch[32];
    const int lp = blockIdx.x;
    DevState* st = B.st + lp;
    if (st->done) return;
    const int c0 = B.cols.first[lp], nc = B.cols.first[lp + 1] - c0;
    const int r0 = B.rows.first[lp], nr = B.rows.first[lp + 1] - r0;
    const double row_max = reduce_partials(partials + SLOT_ROW_MAX * kMaxTiles + r0, nr, scratch, OpMax());
    const double row_dobj = reduce_partials(partials + SLOT_ROW_DOBJ * kMaxTiles + r0, nr, scratch, OpSum());
    const double bad_r = reduce_partials(partials + SLOT_NAN * kMaxTiles + r0, nr, scratch, OpSum());
    const double col_max = reduce_partials(partials + SLOT_COL_MAX * kMaxTiles + c0, nc, scratch, OpMax());
    const double col_dres = reduce_partials(partials + SLOT_COL_DRES * kMaxTiles + c0, nc, scratch, OpSum());
    const double col_pobj = reduce_partials(partials + SLOT_COL_POBJ * kMaxTiles + c0, nc, scratch, OpSum());
    const double col_dobj = reduce_partials(partials + SLOT_COL_DOBJ * kMaxTiles + c0, nc, scratch, OpSum());
    const double bad_c = reduce_partials(partials + SLOT_B * kMaxTiles + c0, nc, scratch, OpSum());
    const double ray_l = reduce_partials(partials + SLOT_RAY_L * kMaxTiles + c0, nc, scratch, OpSum());
    const double ray_cs = reduce_partials(partials + SLOT_RAY_CSCALE * kMaxTiles + c0, nc, scratch, OpSum());
    const double ray_ci = reduce_partials(partials + SLOT_RAY_CINF * kMaxTiles + c0, nc, scratch, OpSum());
    const double ray_rs = reduce_partials(partials + SLOT_RAY_RSCALE * kMaxTiles + r0, nr, scratch, OpSum());
    const double ray_ri = reduce_partials(partials + SLOT_RAY_RINF * kMaxTiles + r0, nr, scratch, OpSum());
    const double ray_u = reduce_partials(partials + SLOT_RAY_U * kMaxTiles + r0, nr, scratch, OpSum());
    if (threadIdx.x != 0) return;
    const double offset = B.offset[lp];
    // the Farkas test of the ray candidate (RayTerms)
    const double margin = ray_l - ray_u;
    const bool farkas = ray_ci == 0.0 && ray_ri == 0.0 && margin > 0.0 && margin > 1e-9 * (ray_cs + ray_rs);
    const double primal = maxv(row_max, col_max);
    const double dual = sqrt(col_dres) / st->c_scale;
    const double pobj = offset + col_pobj;
    const double dobj = (offset + row_dobj) + col_dobj;
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double score = maxv(maxv(primal, dual), gap);
    st->primal_infeas = primal;
    st->dual_infeas = dual;
    st->gap = gap;
    st->objective = pobj;
    st->dual_objective = dobj;
    st->score = score;
    st->restart_pending = 0;
    const long long isr = st->iters_since_restart + span;
    if (bad_r + bad_c > 0.0 || !isfinite(score)) {
        st->nonfinite = 1;
        st->done = 1;
        st->status = 3;
    } else if (!final_pass && primal <= ctl.primal_tol && dual <= ctl.dual_tol && gap <= ctl.gap_tol) {
        st->done = 1;
        st->status = 0;
    } else if (farkas) {
        st->done = 1;
        st->status = 2;           // infeasible_or_unbounded, the dual average is the ray
        st->cert = MC_CERT_DUAL_RAY;
    } else if (!final_pass) {
        const bool do_restart =
            ctl.strategy == 2 ||
            (ctl.strategy == 1 && (score <= ctl.restart_reduction * st->last_restart_score ||
                                   (isr >= 5 * ctl.restart_every && score < st->last_restart_score)));
        if (do_restart) {
            if (ctl.adaptive_weight && primal > 1e-12 && dual > 1e-12) {
                const double ratio = clampv(sqrt(primal / dual), 0.05, 20.0);
                st->omega = clampv(st->omega * pow(ratio, ctl.weight_smoothing), 1e-6, 1e6);
            }
            st->restart_pending = 1;
            st->avg_count = 0;
            st->iters_since_restart = 0;
            st->last_restart_score = score;
            st->restarts += 1;
        } else {
            st->avg_count += span;
            st->iters_since_restart = isr;
        }
    }
    st->iter += span;
    if (!final_pass) st->checks += 1;
}

// restart to the average, over the running tiles (columns, then rows)
__global__ void __launch_bounds__(kBlock) kb_restart_copy(Iterates<double> P, BatchRefs B) {
    const int nc = B.active_count[0], nr = B.active_count[1];
    for (int q = blockIdx.x; q < nc + nr; q += gridDim.x) {
        const bool col = q < nc;
        const int t = col ? B.active[q] : B.active[kMaxTiles + q - nc];
        const TileTable& T = col ? B.cols : B.rows;
        const DevState* st = B.st + T.lp[t];
        if (!st->restart_pending || st->done) continue;
        for (int l = T.l0[t] + threadIdx.x; l < T.l1[t]; l += blockDim.x) {
            if (col) P.x[l] = P.x_avg[l];
            else P.y[l] = P.y_avg[l];
        }
    }
}

// ------------------------------------------------------------------ setup
// Ruiz per LP: line maxima of a tile, per-LP check, deltas and rescale skip
// LPs whose Ruiz has converged (ruiz_scaling.cpp:167-218 per LP).
__global__ void kb_ruiz_line_max(const int* __restrict__ start, const double* __restrict__ value,
                                 double* __restrict__ norm, double* __restrict__ partials, int slot,
                                 TileTable T, const DevState* __restrict__ st) {
    __shared__ double scratch[32];
    double err = 0.0;
    if (!st[T.lp[blockIdx.x]].ruiz_done) {
        for (int j = T.l0[blockIdx.x] + threadIdx.x; j < T.l1[blockIdx.x]; j += blockDim.x) {
            double mx = 0.0;
            for (int p = start[j]; p < start[j + 1]; ++p) mx = maxv(mx, fabs(value[p]));
            if (mx == 0.0) mx = 1.0;
            norm[j] = mx;
            err = maxv(err, fabs(1.0 - mx));
        }
    }
    err = block_reduce(err, scratch, OpMax());
    if (threadIdx.x == 0) partials[slot * kMaxTiles + blockIdx.x] = err;
}

__global__ void kb_ruiz_check(const double* __restrict__ partials, BatchRefs B, double tolerance) {
    __shared__ double scratch[32];
    const int lp = blockIdx.x;
    DevState* st = B.st + lp;
    if (st->ruiz_done) return;
    const int c0 = B.cols.first[lp], nc = B.cols.first[lp + 1] - c0;
    const int r0 = B.rows.first[lp], nr = B.rows.first[lp + 1] - r0;
    const double c = reduce_partials(partials + SLOT_A * kMaxTiles + c0, nc, scratch, OpMax());
    const double r = reduce_partials(partials + SLOT_B * kMaxTiles + r0, nr, scratch, OpMax());
    if (threadIdx.x == 0) {
        if (r < tolerance && c < tolerance) st->ruiz_done = 1;
        else st->ruiz_passes += 1;
    }
}

__global__ void kb_ruiz_deltas(double* __restrict__ norm, double* __restrict__ scale, TileTable T,
                               const DevState* __restrict__ st) {
    if (st[T.lp[blockIdx.x]].ruiz_done) return;
    for (int j = T.l0[blockIdx.x] + threadIdx.x; j < T.l1[blockIdx.x]; j += blockDim.x) {
        const double d = 1.0 / sqrt(norm[j]);
        norm[j] = d;
        scale[j] *= d;
    }
}

__global__ void kb_ruiz_rescale(const int* __restrict__ start, const int* __restrict__ inner,
                                double* __restrict__ value, const double* __restrict__ delta_outer,
                                const double* __restrict__ delta_inner, TileTable T,
                                const DevState* __restrict__ st) {
    if (st[T.lp[blockIdx.x]].ruiz_done) return;
    for (int j = T.l0[blockIdx.x] + threadIdx.x; j < T.l1[blockIdx.x]; j += blockDim.x) {
        const double dout = delta_outer[j];
        for (int p = start[j]; p < start[j + 1]; ++p)
            value[p] = __dmul_rn(value[p], __dmul_rn(delta_inner[inner[p]], dout));
    }
}

// Column setup of a tile (k_setup_cols per LP) plus the crossed-bound
// certificate: a column with lower > upper makes its LP infeasible.
__global__ void kb_setup_cols(const int* __restrict__ col_start, const double* __restrict__ value,
                              const double* __restrict__ obj_in, const double* __restrict__ lo_in,
                              const double* __restrict__ hi_in, const double* __restrict__ col_scale,
                              const double* __restrict__ obj_sign, Iterates<double> P, Original O,
                              double* __restrict__ partials, BatchRefs B) {
    __shared__ double scratch[32];
    const int lp = B.cols.lp[blockIdx.x];
    const double sign = obj_sign[lp];
    double cmax = 0.0, comax = 0.0;
    int crossed = 0;
    for (int j = B.cols.l0[blockIdx.x] + threadIdx.x; j < B.cols.l1[blockIdx.x]; j += blockDim.x) {
        const double s = col_scale[j];
        const double inv = 1.0 / s;
        const double l0 = lo_in[j], h0 = hi_in[j];
        const double ls = isfinite(l0) ? __dmul_rn(l0, inv) : l0;
        const double hs = isfinite(h0) ? __dmul_rn(h0, inv) : h0;
        const double lsent = isinf(ls) ? -kBig : ls;
        const double hsent = isinf(hs) ? kBig : hs;
        const_cast<double*>(P.lo)[j] = lsent;
        const_cast<double*>(P.hi)[j] = hsent;
        const_cast<double*>(O.lo)[j] = isinf(l0) ? -kBig : l0;
        const_cast<double*>(O.hi)[j] = isinf(h0) ? kBig : h0;
        if (l0 > h0 && !crossed) {
            crossed = 1;
            atomicMin(B.cert_idx + lp, j - B.cols.l0[B.cols.first[lp]]);
        }
        const double cj = sign * __dmul_rn(obj_in[j], s);
        const_cast<double*>(P.c)[j] = cj;
        cmax = maxv(cmax, fabs(cj));
        const double co = sign * obj_in[j];
        const_cast<double*>(O.c)[j] = co;
        comax = maxv(comax, fabs(co));
        double nrm = 0.0;
        for (int p = col_start[j]; p < col_start[j + 1]; ++p) nrm += fabs(value[p]);
        const_cast<double*>(P.col_norm)[j] = (nrm < 1e-12) ? 1.0 : nrm;
        // start as k_setup_cols: the caller's point scaled into the
        // equilibrated space and projected, else proj(0)
        const double start = (B.warm && (B.warm[lp] & 1)) ? __dmul_rn(B.warm_x[j], inv) : 0.0;
        const double x0 = clampv(start, lsent, hsent);
        P.x[j] = x0;
        P.x_avg[j] = x0;
    }
    if (crossed) atomicOr(B.flags + lp, 1);
    cmax = block_reduce(cmax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_A * kMaxTiles + blockIdx.x] = cmax;
    comax = block_reduce(comax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_B * kMaxTiles + blockIdx.x] = comax;
}

// Row setup of a tile (k_setup_rows per LP) plus the row-activity
// certificate: with every variable in its (original) box a row's activity
// lies in [sum min(a l, a u), sum max(a l, a u)]; if that interval misses the
// row's [b_lo, b_hi] (beyond a relative 1e-9) the LP is infeasible.
__global__ void kb_setup_rows(const int* __restrict__ row_start, const int* __restrict__ col_index,
                              const double* __restrict__ value, const double* __restrict__ rlo_in,
                              const double* __restrict__ rhi_in, const double* __restrict__ row_scale,
                              const double* __restrict__ col_scale, const double* __restrict__ lo_in,
                              const double* __restrict__ hi_in, Iterates<double> P, Original O,
                              double* __restrict__ partials, BatchRefs B) {
    __shared__ double scratch[32];
    const int lp = B.rows.lp[blockIdx.x];
    double bmax = 0.0;
    int infeasible = 0;
    for (int i = B.rows.l0[blockIdx.x] + threadIdx.x; i < B.rows.l1[blockIdx.x]; i += blockDim.x) {
        const double s = row_scale[i];
        const double l0 = rlo_in[i], h0 = rhi_in[i];
        const double ls = isfinite(l0) ? __dmul_rn(l0, s) : l0;
        const double hs = isfinite(h0) ? __dmul_rn(h0, s) : h0;
        const double lsent = isinf(ls) ? -kBig : ls;
        const double hsent = isinf(hs) ? kBig : hs;
        const_cast<double*>(P.blo)[i] = lsent;
        const_cast<double*>(P.bhi)[i] = hsent;
        const_cast<double*>(O.blo)[i] = isinf(l0) ? -kBig : l0;
        const_cast<double*>(O.bhi)[i] = isinf(h0) ? kBig : h0;
        if (fabs(lsent) < 1e299) bmax = maxv(bmax, fabs(lsent));
        if (fabs(hsent) < 1e299) bmax = maxv(bmax, fabs(hsent));
        double nrm = 0.0, amin = 0.0, amax = 0.0, mag = 0.0;
        for (int p = row_start[i]; p < row_start[i + 1]; ++p) {
            nrm += fabs(value[p]);
            // original coefficient and bounds: a = value / (row_scale * col_scale)
            const int j = col_index[p];
            const double a = value[p] / (s * col_scale[j]);
            const double lj = lo_in[j], hj = hi_in[j];
            const double t1 = a * lj, t2 = a * hj;  // +-inf when unbounded
            amin += (a > 0) ? t1 : t2;
            amax += (a > 0) ? t2 : t1;
            mag += fabs(a) * maxv(isfinite(lj) ? fabs(lj) : 0.0, isfinite(hj) ? fabs(hj) : 0.0);
        }
        const_cast<double*>(P.row_norm)[i] = (nrm < 1e-12) ? 1.0 : nrm;
        const double slack = 1e-9 * (1.0 + mag + maxv(isfinite(l0) ? fabs(l0) : 0.0, isfinite(h0) ? fabs(h0) : 0.0));
        if ((isfinite(l0) && amax < l0 - slack) || (isfinite(h0) && amin > h0 + slack)) {
            if (!infeasible) atomicMin(B.cert_idx + B.nlp + lp, i - B.rows.l0[B.rows.first[lp]]);
            infeasible = 1;
        }
        const double y0 = (B.warm && (B.warm[lp] & 2)) ? __dmul_rn(B.warm_y[i], 1.0 / s) : 0.0;
        P.y[i] = y0;
        P.y_avg[i] = y0;
        B.y_prev[i] = y0;
    }
    if (infeasible) atomicOr(B.flags + lp, 2);
    bmax = block_reduce(bmax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_C * kMaxTiles + blockIdx.x] = bmax;
}

// per-LP scalars (k_setup_scalars per LP); an LP with a certificate is
// terminated at once as infeasible_or_unbounded
__global__ void kb_setup_scalars(const double* __restrict__ partials, BatchRefs B, double initial_primal_weight,
                                 double step_size_reduction) {
    __shared__ double scratch[32];
    const int lp = blockIdx.x;
    DevState* st = B.st + lp;
    const int c0 = B.cols.first[lp], nc = B.cols.first[lp + 1] - c0;
    const int r0 = B.rows.first[lp], nr = B.rows.first[lp + 1] - r0;
    const double cmax = reduce_partials(partials + SLOT_A * kMaxTiles + c0, nc, scratch, OpMax());
    const double comax = reduce_partials(partials + SLOT_B * kMaxTiles + c0, nc, scratch, OpMax());
    const double bmax = reduce_partials(partials + SLOT_C * kMaxTiles + r0, nr, scratch, OpMax());
    if (threadIdx.x == 0) {
        const double c_norm = maxv(1.0, cmax);
        const double b_norm = maxv(1.0, bmax);
        st->c_norm_inf = c_norm;
        st->b_norm_inf = b_norm;
        st->c_scale = maxv(1.0, comax);
        st->omega = (initial_primal_weight > 0.0) ? initial_primal_weight
                                                  : clampv(sqrt(c_norm / b_norm), 0.01, 100.0);
        st->eta = clampv(step_size_reduction, 0.1, 0.99);
        st->last_restart_score = 1e300;
        st->primal_infeas = st->dual_infeas = st->gap = 1e300;
        st->iter = 0;
        st->avg_count = 0;
        st->iters_since_restart = 0;
        st->restarts = 0;
        st->checks = 0;
        st->restart_pending = 0;
        st->nonfinite = 0;
        if (B.flags[lp]) {
            st->done = 1;
            st->status = 2;  // infeasible_or_unbounded, certified at setup
            st->cert = (B.flags[lp] & 1) ? MC_CERT_CROSSED_BOUNDS : MC_CERT_ROW_ACTIVITY;
        } else {
            st->done = 0;
            st->status = 1;
            st->cert = MC_CERT_NONE;
        }
    }
}

// per-tile unscaled output (k_unscale_out over the tile's lines): x = x_avg
// D_C, y = y_avg D_R; in the mixed form the averages are the FP64 base plus
// the FP32 average correction (dx_avg, dy_avg non-null)
__global__ void kb_unscale_out(const double* __restrict__ x_avg, const float* __restrict__ dx_avg,
                               const double* __restrict__ y_avg, const float* __restrict__ dy_avg,
                               const double* __restrict__ col_scale, const double* __restrict__ row_scale,
                               double* __restrict__ x_out, double* __restrict__ y_out, BatchRefs B) {
    const bool col = blockIdx.x < (unsigned)B.cols.ntiles;
    const int t = col ? blockIdx.x : blockIdx.x - B.cols.ntiles;
    const TileTable& T = col ? B.cols : B.rows;
    // an LP proven infeasible by a dual ray returns the ray as its dual
    const DevState& S = B.st[T.lp[t]];
    const bool ray = S.status == 2 && S.cert == MC_CERT_DUAL_RAY;
    for (int l = T.l0[t] + threadIdx.x; l < T.l1[t]; l += blockDim.x) {
        if (col) x_out[l] = __dmul_rn(dx_avg ? x_avg[l] + (double)dx_avg[l] : x_avg[l], col_scale[l]);
        else if (ray) y_out[l] = __dmul_rn(B.dray[l], row_scale[l]);
        else y_out[l] = __dmul_rn(dy_avg ? y_avg[l] + (double)dy_avg[l] : y_avg[l], row_scale[l]);
    }
}

// shift a packed LP's CSC indices into the packed numbering
__global__ void kb_shift_indices(int* __restrict__ col_start, int* __restrict__ row_index, int ncols, long long nnz,
                                 int nnz_offset, int row_offset) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nnz + ncols;
         t += (long long)gridDim.x * blockDim.x) {
        if (t < nnz) row_index[t] += row_offset;
        else col_start[t - nnz] += nnz_offset;
    }
}

// The work queue, rebuilt after every check in two launches.  An LP's tiles
// are contiguous and an LP is either running or done, so the running tiles
// are the tile ranges of the running LPs, in LP order:
//   kb_compact (one block): offsets of each LP's range in the two lists (an
//     exclusive scan over the LPs), the list lengths, and the packed loop's
//     poll flag (done once every LP is done);
//   kb_fill_active (one thread per tile): a running LP's tile t goes to
//     position offset(LP) + (t - first tile of the LP).
constexpr int kCompactThreads = 1024;

__global__ void __launch_bounds__(kCompactThreads) kb_compact(BatchRefs B, int* __restrict__ lp_offset,
                                                              int* __restrict__ active_count,
                                                              DevState* __restrict__ global) {
    __shared__ int warp_total[32];
    __shared__ int base;
    __shared__ int running;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kCompactThreads / 32;
    if (threadIdx.x == 0) running = 0;
    for (int which = 0; which < 2; ++which) {
        const TileTable& T = which ? B.rows : B.cols;
        int* off = lp_offset + which * (B.nlp + 1);
        if (threadIdx.x == 0) base = 0;
        __syncthreads();
        for (int b0 = 0; b0 < B.nlp; b0 += kCompactThreads) {
            const int b = b0 + threadIdx.x;
            const bool run = b < B.nlp && !B.st[b].done;
            const int cnt = run ? T.first[b + 1] - T.first[b] : 0;
            if (which == 0 && run) atomicAdd(&running, 1);
            int v = cnt;  // inclusive scan within the warp
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, d);
                if (lane >= d) v += u;
            }
            if (lane == 31) warp_total[warp] = v;
            __syncthreads();
            if (warp == 0) {
                int w = warp_total[lane];
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, w, d);
                    if (lane >= d) w += u;
                }
                warp_total[lane] = w;  // inclusive prefix over warps
            }
            __syncthreads();
            const int excl = base + (warp ? warp_total[warp - 1] : 0) + v - cnt;
            if (b < B.nlp) off[b] = excl;
            __syncthreads();
            if (threadIdx.x == 0) base += warp_total[kWarps - 1];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            off[B.nlp] = base;
            active_count[which] = base;
            global->active_tiles[which] = base;  // read by the host's poll
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) global->done = running == 0 ? 1 : 0;
}

__global__ void __launch_bounds__(kBlock) kb_fill_active(BatchRefs B, const int* __restrict__ lp_offset,
                                                         int* __restrict__ active) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= B.cols.ntiles + B.rows.ntiles) return;
    const int which = q < B.cols.ntiles ? 0 : 1;
    const int t = which ? q - B.cols.ntiles : q;
    const TileTable& T = which ? B.rows : B.cols;
    const int lp = T.lp[t];
    if (B.st[lp].done) return;
    active[which * kMaxTiles + lp_offset[which * (B.nlp + 1) + lp] + (t - T.first[lp])] = t;
}

// ------------------------------------------------- mixed precision, batched
// The FP32 + FP64-refinement form (mixed.cuh) per LP: the correction LP of
// every LP is iterated in FP32 over the packed FP32 matrix, its residuals,
// restart and termination are evaluated in FP64, and at each restart of an LP
// its base moves to the average and its correction data are rebuilt.

template <int G>
__global__ void __launch_bounds__(kBlock, kMixedRowBlocks) kb_dual_mx(Iterates<float> P, MixedState M, BatchRefs B, int k) {
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 1, t) {
        const DevState* st = B.st + B.rows.lp[t];
        const float sg = (float)(st->eta * st->omega);
        const float cnt = (float)(double)(st->avg_count + k + 1);
        MC_TILE_LINES(B.rows, t, i, valid, sub) {
            const bool owner = valid && sub == 0;
            float rn = 1.f, dy = 0.f, dya = 0.f, yb = 0.f, rl = 0.f, rh = 0.f;
            if (owner) {
                rn = ld_stream(P.row_norm + i);
                dy = ld_stream(P.y + i);
                dya = ld_stream(P.y_avg + i);
                yb = ld_stream(M.yb + i);
                rl = ld_stream(M.r_lo + i);
                rh = ld_stream(M.r_hi + i);
            }
            const float ax = line_dot<G>(P.csr_start, P.csr_col, P.csr_val, P.x_bar, i, valid, sub, pol);
            if (owner) dual_update_mx(P, M, i, ax, sg, cnt, pol, rn, dy, dya, yb, rl, rh);
        }
    }
}

__global__ void __launch_bounds__(kBlock) kb_dual_apply_mx(Iterates<float> P, MixedState M, BatchRefs B, int k) {
    const unsigned long long pol = policy_keep();
    MC_FOR_ACTIVE(B, 1, t) {
        const DevState* st = B.st + B.rows.lp[t];
        const float sg = (float)(st->eta * st->omega);
        const float cnt = (float)(double)(st->avg_count + k + 1);
        for (int i = B.rows.l0[t] + threadIdx.x; i < B.rows.l1[t]; i += blockDim.x)
            dual_update_mx(P, M, i, P.ax_bar[i], sg, cnt, pol, ld_stream(P.row_norm + i), ld_stream(P.y + i),
                           ld_stream(P.y_avg + i), ld_stream(M.yb + i), ld_stream(M.r_lo + i),
                           ld_stream(M.r_hi + i));
    }
}

// FP64 residual pass of each running LP on x_hat + dx_avg, y_hat + dy_avg,
// keeping A x and A^T y of that point for the recentring.
template <int G>
__global__ void __launch_bounds__(kBlock) kb_residual_rows_mx(Iterates<float> P, MixedState M, Original O,
                                                              BatchRefs B) {
    __shared__ double scratch[32];
    MC_FOR_ACTIVE(B, 1, t) {
        RowTerms acc;
        RayTerms ray;
        MC_TILE_LINES(B.rows, t, i, valid, sub) {
            double s = 0.0;
            if (valid) {
                const int b = P.csr_start[i], e = P.csr_start[i + 1];
                for (int p = b + sub; p < e; p += G) {
                    const int jj = P.csr_col[p];
                    s = fma(M.csr_val64[p], M.x_hat[jj] + (double)P.x_avg[jj], s);
                }
            }
            s = group_sum<G>(s);
            if (valid && sub == 0) {
                M.ax_full[i] = s;
                const double yv = M.y_hat[i] + (double)P.y_avg[i];
                acc.add(O, i, s, yv);
                const double d = RayTerms::candidate(O, i, yv, B.y_prev + i);
                B.dray[i] = d;
                ray.add_row(O, i, d);
            }
        }
        acc.vmax = block_reduce(acc.vmax, scratch, OpMax());
        acc.dsum = block_reduce(acc.dsum, scratch, OpSum());
        acc.bad = block_reduce(acc.bad, scratch, OpSum());
        if (threadIdx.x == 0) {
            P.partials[SLOT_ROW_MAX * kMaxTiles + t] = acc.vmax;
            P.partials[SLOT_ROW_DOBJ * kMaxTiles + t] = acc.dsum;
            P.partials[SLOT_NAN * kMaxTiles + t] = acc.bad;
        }
        ray.store_rows(P.partials, scratch, t);
    }
}

template <int G>
__global__ void __launch_bounds__(kBlock) kb_residual_cols_mx(Iterates<float> P, MixedState M, Original O,
                                                              BatchRefs B) {
    __shared__ double scratch[32];
    MC_FOR_ACTIVE(B, 0, t) {
        ColTerms acc;
        RayTerms ray;
        MC_TILE_LINES(B.cols, t, j, valid, sub) {
            double s = 0.0, sd = 0.0, sa = 0.0;
            if (valid) {
                const int b = P.csc_start[j], e = P.csc_start[j + 1];
                for (int p = b + sub; p < e; p += G) {
                    const int ii = P.csc_row[p];
                    const double a = M.csc_val64[p], dv = B.dray[ii];
                    s = fma(a, M.y_hat[ii] + (double)P.y_avg[ii], s);
                    sd = fma(a, dv, sd);
                    sa = fma(fabs(a), fabs(dv), sa);
                }
            }
            s = group_sum<G>(s);
            sd = group_sum<G>(sd);
            sa = group_sum<G>(sa);
            if (valid && sub == 0) {
                M.aty_full[j] = s;
                acc.add(O, j, s, M.x_hat[j] + (double)P.x_avg[j]);
                ray.add_col(O, j, sd, sa);
            }
        }
        acc.vmax = block_reduce(acc.vmax, scratch, OpMax());
        acc.dres = block_reduce(acc.dres, scratch, OpSum());
        acc.pobj = block_reduce(acc.pobj, scratch, OpSum());
        acc.dobj = block_reduce(acc.dobj, scratch, OpSum());
        acc.bad = block_reduce(acc.bad, scratch, OpSum());
        if (threadIdx.x == 0) {
            P.partials[SLOT_COL_MAX * kMaxTiles + t] = acc.vmax;
            P.partials[SLOT_COL_DRES * kMaxTiles + t] = acc.dres;
            P.partials[SLOT_COL_POBJ * kMaxTiles + t] = acc.pobj;
            P.partials[SLOT_COL_DOBJ * kMaxTiles + t] = acc.dobj;
            P.partials[SLOT_B * kMaxTiles + t] = acc.bad;
        }
        ray.store_cols(P.partials, scratch, t);
    }
}

// Restart of an LP to its average in the mixed form: its base moves there and
// its correction LP's data are rebuilt from the residual pass's FP64 products
// (k_recenter_mx per LP).  `force` rebuilds every running LP (the start).
__global__ void __launch_bounds__(kBlock) kb_recenter_mx(Iterates<float> P, MixedState M, BatchRefs B, int force) {
    const float inf = __int_as_float(0x7f800000);
    const int nc = B.active_count[0], nr = B.active_count[1];
    for (int q = blockIdx.x; q < nc + nr; q += gridDim.x) {
        const bool col = q < nc;
        const int t = col ? B.active[q] : B.active[kMaxTiles + q - nc];
        const TileTable& T = col ? B.cols : B.rows;
        const DevState* st = B.st + T.lp[t];
        if (st->done || (!force && !st->restart_pending)) continue;
        for (int l = T.l0[t] + threadIdx.x; l < T.l1[t]; l += blockDim.x) {
            if (col) {
                const double xh = M.x_hat[l] + (double)P.x_avg[l];
                M.x_hat[l] = xh;
                P.x[l] = 0.f;
                P.x_avg[l] = 0.f;
                M.g[l] = (float)(M.c64[l] + M.aty_full[l]);
                const double lo = M.lo64[l], hi = M.hi64[l];
                M.lo[l] = (lo <= -1e299) ? -inf : (float)(lo - xh);
                M.hi[l] = (hi >= 1e299) ? inf : (float)(hi - xh);
            } else {
                const double yh = M.y_hat[l] + (double)P.y_avg[l];
                M.y_hat[l] = yh;
                P.y[l] = 0.f;
                P.y_avg[l] = 0.f;
                M.yb[l] = (float)yh;
                const double ax = M.ax_full[l], lo = M.blo64[l], hi = M.bhi64[l];
                M.r_lo[l] = (lo <= -1e299) ? inf : (float)(ax - lo);
                M.r_hi[l] = (hi >= 1e299) ? -inf : (float)(ax - hi);
            }
        }
    }
}

#undef MC_TILE_LINES
#undef MC_FOR_ACTIVE

}  // namespace mc
