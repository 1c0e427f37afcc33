// Variants of one LP that differ only in their variable bounds, solved
// together with the matrix read once per iteration for all of them (included
// once, by engine.cu after batch.cuh).
//
// Branch and bound creates such LPs: every node of a round is the parent LP
// with a few bounds tightened (src/milp/milp_solver.cpp:401-447).  Packing K
// copies block-diagonally (batch.cuh) streams the matrix K times per
// iteration and turns every nonzero into K random 8-byte gathers.  Here the
// iterates are stored variant-minor -- element (j, k) of an n x K array at
// j * Kp + k, Kp = K rounded up to 32 -- and one warp carries 32 variants of
// a line: a nonzero a_ij is loaded once per warp (a broadcast) and the
// gathered vector entry for 32 variants is one contiguous 256-byte read.
//
// Every variant still runs the reference algorithm on its own
// (src/lp/first_order/pdlp.cpp:139-276): own step size, primal weight,
// restarts and termination, from its own DevState.  The shared setup (Ruiz
// scaling, norms, c, row bounds, the initial primal weight) depends only on
// A, c and the row bounds, which the variants share; their bounds are scaled
// and projected per variant.  Reductions are per variant: each block writes
// one partial per variant and a per-variant kernel sums them in a fixed
// order, so results are run-to-run deterministic.  Infeasible variants are
// certified as in the packed batch (crossed bounds, row activity, and the
// Farkas test of the dual ray candidate at every restart check).
#pragma once

#include "batch.cuh"

namespace mc {

constexpr int kVarWarps = kBlock / 32;  // warps per block, one line each per trip

// The base LP (scaled, shared by every variant).
struct VarBase {
    int m, n;
    const int* cs;        // CSC of the scaled A
    const int* ri;
    const double* cv;
    const int* rs;        // CSR of the scaled A
    const int* ci;
    const double* rv;
    const double* c;      // scaled objective (minimisation sign)
    const double* col_norm;
    const double* row_norm;
    const double* blo;    // scaled row bounds, sentinel form
    const double* bhi;
};

// The per-variant arrays (variant-minor, row stride Kp).
struct VarRefs {
    int K, Kp, nb;         // variants, padded count, blocks per grid row (partials per variant)
    DevState* st;          // [K]
    DevState* global;      // poll flag: every variant done
    double* lo;            // [n Kp] scaled bounds, sentinel form
    double* hi;
    double* olo;           // [n Kp] original bounds, sentinel form
    double* ohi;
    double* x;             // [n Kp]
    double* xb;            // [n Kp] x-bar (non-step iterations)
    double* xa;            // [n Kp] average
    double* xdx;           // [2 n Kp] (x-bar, dx) pairs (step-size iterations)
    double* y;             // [m Kp]
    double* ya;
    double* axb;           // [m Kp] A x-bar of a step-size iteration
    double* y_prev;        // [m Kp] dual average at the previous check (the start at setup)
    double* dray;          // [m Kp] the dual ray candidate of the current check
    double* partials;      // [NUM_SLOTS Kp nb]
    int* flags;            // [K] setup certificates: 1 crossed bounds, 2 row activity
    int* cert_idx;         // [2K] lowest crossed column, lowest failing row (INT_MAX if none)
};

__device__ __forceinline__ double* var_partial(const VarRefs& V, int slot, int k) {
    return V.partials + ((size_t)slot * V.Kp + k) * V.nb;
}

// Sum (or max) of one value per lane over the block's warps, in warp order;
// the result is valid in warp 0 (lane = variant).  Ends with a barrier.
template <class Op>
__device__ __forceinline__ double lanes_reduce(double v, double (*sm)[33], Op op) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    sm[warp][lane] = v;
    __syncthreads();
    if (warp == 0)
        for (int w = 1; w < kVarWarps; ++w) v = op(v, sm[w][lane]);
    __syncthreads();
    return v;
}

// The lane's variant; `live` when it exists and still runs.  Every block
// works on one group of 32 variants (blockIdx.y), so a block whose variants
// have all finished leaves as a whole.
#define MC_VARIANT_LANE(V, K_, LIVE)                                   \
    const int lane_ = threadIdx.x & 31;                                \
    const int K_ = blockIdx.y * 32 + lane_;                            \
    const bool LIVE = K_ < (V).K && !(V).st[K_].done;                  \
    if (!__syncthreads_or(LIVE)) return;

// Lines of the block's warps: line = blockIdx.x * warps + warp, strided over the grid.
#define MC_VARIANT_LINES(LINE, COUNT)                                                            \
    for (long long LINE = (long long)blockIdx.x * kVarWarps + (threadIdx.x >> 5); LINE < (COUNT); \
         LINE += (long long)gridDim.x * kVarWarps)

// Dot of CSR/CSC line `l` with the variant-minor vector v (column k), four
// gathers in flight; inactive lanes issue no loads.
__device__ __forceinline__ double variant_dot(const int* __restrict__ start, const int* __restrict__ idx,
                                              const double* __restrict__ val, const double* __restrict__ v,
                                              int Kp, long long l, int k, bool live, unsigned long long pol) {
    const int b = __ldg(start + l), e = __ldg(start + l + 1);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int p = b;
    for (; p + 4 <= e; p += 4) {
        const int i0 = __ldg(idx + p), i1 = __ldg(idx + p + 1), i2 = __ldg(idx + p + 2), i3 = __ldg(idx + p + 3);
        const double a0 = __ldg(val + p), a1 = __ldg(val + p + 1), a2 = __ldg(val + p + 2), a3 = __ldg(val + p + 3);
        if (live) {
            s0 = fma(a0, ld_keep(v + (size_t)i0 * Kp + k, pol), s0);
            s1 = fma(a1, ld_keep(v + (size_t)i1 * Kp + k, pol), s1);
            s2 = fma(a2, ld_keep(v + (size_t)i2 * Kp + k, pol), s2);
            s3 = fma(a3, ld_keep(v + (size_t)i3 * Kp + k, pol), s3);
        }
    }
    for (; p < e; ++p)
        if (live) s0 = fma(__ldg(val + p), ld_keep(v + (size_t)__ldg(idx + p) * Kp + k, pol), s0);
    return (s0 + s1) + (s2 + s3);
}

// ------------------------------------------------------------------ primal
// g = c + A^T y; x+ = clamp(x - tau g, l, u); x-bar; average; on step-size
// iterations dx and sum col_norm dx^2 per variant (pdlp.cpp:195-206, :226)
template <bool STEP>
__global__ void __launch_bounds__(kBlock) kv_primal(VarBase Bs, VarRefs V, int kk) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    double step = 0.0, cnt = 1.0;
    if (live) {
        const DevState& s = V.st[k];
        step = s.eta / s.omega;
        cnt = (double)(s.avg_count + kk + 1);
    }
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    MC_VARIANT_LINES(j, Bs.n) {
        const double aty = variant_dot(Bs.cs, Bs.ri, Bs.cv, V.y, V.Kp, j, k, live, pol);
        if (live) {
            const size_t q = (size_t)j * V.Kp + k;
            const double cn = __ldg(Bs.col_norm + j);
            const double g = __dadd_rn(__ldg(Bs.c + j), aty);
            const double tau = __ddiv_rn(step, cn);
            const double xo = ld_stream(V.x + q);
            const double xp = clampv(__dsub_rn(xo, __dmul_rn(tau, g)), ld_stream(V.lo + q), ld_stream(V.hi + q));
            const double d = __dsub_rn(xp, xo);
            const double xbar = __dsub_rn(__dmul_rn(2.0, xp), xo);
            if (STEP) {
                st_keep2(V.xdx + 2 * q, xbar, d, pol);
                acc += __dmul_rn(__dmul_rn(cn, d), d);
            } else {
                st_keep(V.xb + q, xbar, pol);
            }
            st_stream(V.x + q, xp);
            const double xa = ld_stream(V.xa + q);
            st_stream(V.xa + q, __dadd_rn(xa, __ddiv_rn(__dsub_rn(xp, xa), cnt)));
        }
    }
    if (STEP) {
        acc = lanes_reduce(acc, sm, OpSum());
        if ((threadIdx.x >> 5) == 0 && k < V.K) var_partial(V, SLOT_DX, k)[blockIdx.x] = acc;
    }
}

// ------------------------------------------------------------------- dual
__device__ __forceinline__ void variant_dual_update(const VarBase& Bs, const VarRefs& V, long long i, int k,
                                                    double ax, double sg, double cnt, unsigned long long pol) {
    const size_t q = (size_t)i * V.Kp + k;
    const double sigma = __ddiv_rn(sg, __ldg(Bs.row_norm + i));
    const double v = __dadd_rn(ld_stream(V.y + q), __dmul_rn(sigma, ax));
    const double yn =
        __dsub_rn(v, __dmul_rn(sigma, clampv(__ddiv_rn(v, sigma), __ldg(Bs.blo + i), __ldg(Bs.bhi + i))));
    st_keep(V.y + q, yn, pol);
    const double ya = ld_stream(V.ya + q);
    st_stream(V.ya + q, __dadd_rn(ya, __ddiv_rn(__dsub_rn(yn, ya), cnt)));
}

// v = y + sigma (A x-bar); y+ = v - sigma clamp(v/sigma, b_lo, b_hi); average (pdlp.cpp:220-227)
__global__ void __launch_bounds__(kBlock) kv_dual(VarBase Bs, VarRefs V, int kk) {
    MC_VARIANT_LANE(V, k, live);
    double sg = 0.0, cnt = 1.0;
    if (live) {
        const DevState& s = V.st[k];
        sg = s.eta * s.omega;
        cnt = (double)(s.avg_count + kk + 1);
    }
    const unsigned long long pol = policy_keep();
    MC_VARIANT_LINES(i, Bs.m) {
        const double ax = variant_dot(Bs.rs, Bs.ci, Bs.rv, V.xb, V.Kp, i, k, live, pol);
        if (live) variant_dual_update(Bs, V, i, k, ax, sg, cnt, pol);
    }
}

// Step-size iteration: A x-bar (kept) and A dx from the (x-bar, dx) pairs,
// sum (A dx)_i^2 / row_norm_i per variant (pdlp.cpp:207-210)
__global__ void __launch_bounds__(kBlock) kv_dual_probe(VarBase Bs, VarRefs V) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    MC_VARIANT_LINES(i, Bs.m) {
        const int b = __ldg(Bs.rs + i), e = __ldg(Bs.rs + i + 1);
        double sv0 = 0.0, sw0 = 0.0, sv1 = 0.0, sw1 = 0.0;
        int p = b;
        for (; p + 2 <= e; p += 2) {
            const int j0 = __ldg(Bs.ci + p), j1 = __ldg(Bs.ci + p + 1);
            const double a0 = __ldg(Bs.rv + p), a1 = __ldg(Bs.rv + p + 1);
            if (live) {
                double v0, w0, v1, w1;
                ld_keep2(V.xdx + 2 * ((size_t)j0 * V.Kp + k), pol, v0, w0);
                ld_keep2(V.xdx + 2 * ((size_t)j1 * V.Kp + k), pol, v1, w1);
                sv0 = fma(a0, v0, sv0);
                sw0 = fma(a0, w0, sw0);
                sv1 = fma(a1, v1, sv1);
                sw1 = fma(a1, w1, sw1);
            }
        }
        if (p < e && live) {
            double v0, w0;
            ld_keep2(V.xdx + 2 * ((size_t)__ldg(Bs.ci + p) * V.Kp + k), pol, v0, w0);
            const double a0 = __ldg(Bs.rv + p);
            sv0 = fma(a0, v0, sv0);
            sw0 = fma(a0, w0, sw0);
        }
        if (live) {
            V.axb[(size_t)i * V.Kp + k] = sv0 + sv1;
            const double adx = sw0 + sw1;
            acc += __ddiv_rn(__dmul_rn(adx, adx), __ldg(Bs.row_norm + i));
        }
    }
    acc = lanes_reduce(acc, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) var_partial(V, SLOT_ADX, k)[blockIdx.x] = acc;
}

// The adaptive eta rule per variant (pdlp.cpp:207-219), one block per variant.
__global__ void kv_step_size(VarRefs V, Controls ctl) {
    __shared__ double scratch[32];
    const int k = blockIdx.x;
    DevState* st = V.st + k;
    if (st->done) return;
    const double dxn = reduce_partials(var_partial(V, SLOT_DX, k), V.nb, scratch, OpSum());
    const double adx = reduce_partials(var_partial(V, SLOT_ADX, k), V.nb, scratch, OpSum());
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

// Step-size iteration: the dual update from the kept A x-bar.
__global__ void __launch_bounds__(kBlock) kv_dual_apply(VarBase Bs, VarRefs V, int kk) {
    MC_VARIANT_LANE(V, k, live);
    if (!live) return;  // no barrier follows
    const DevState& s = V.st[k];
    const double sg = s.eta * s.omega;
    const double cnt = (double)(s.avg_count + kk + 1);
    const unsigned long long pol = policy_keep();
    MC_VARIANT_LINES(i, Bs.m) variant_dual_update(Bs, V, i, k, V.axb[(size_t)i * V.Kp + k], sg, cnt, pol);
}

// --------------------------------------------------------------- residuals
// compute_unscaled_residuals (pdlp.cpp:62-135) of every variant's averages,
// with the Farkas test terms (RayTerms).
__global__ void __launch_bounds__(kBlock) kv_residual_rows(VarBase Bs, VarRefs V, Original O) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    const unsigned long long pol = policy_keep();
    RowTerms acc;
    RayTerms ray;
    MC_VARIANT_LINES(i, Bs.m) {
        const double s = variant_dot(Bs.rs, Bs.ci, Bs.rv, V.xa, V.Kp, i, k, live, pol);
        if (live) {
            const size_t q = (size_t)i * V.Kp + k;
            const double yv = V.ya[q];
            acc.add(O, (int)i, s, yv);
            const double d = RayTerms::candidate(O, (int)i, yv, V.y_prev + q);
            V.dray[q] = d;
            ray.add_row(O, (int)i, d);
        }
    }
    const double vmax = lanes_reduce(acc.vmax, sm, OpMax());
    const double dsum = lanes_reduce(acc.dsum, sm, OpSum());
    const double bad = lanes_reduce(acc.bad, sm, OpSum());
    const double ru = lanes_reduce(ray.u, sm, OpSum());
    const double rsc = lanes_reduce(ray.rscale, sm, OpSum());
    const double rinf = lanes_reduce(ray.rinf, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) {
        var_partial(V, SLOT_ROW_MAX, k)[blockIdx.x] = vmax;
        var_partial(V, SLOT_ROW_DOBJ, k)[blockIdx.x] = dsum;
        var_partial(V, SLOT_NAN, k)[blockIdx.x] = bad;
        var_partial(V, SLOT_RAY_U, k)[blockIdx.x] = ru;
        var_partial(V, SLOT_RAY_RSCALE, k)[blockIdx.x] = rsc;
        var_partial(V, SLOT_RAY_RINF, k)[blockIdx.x] = rinf;
    }
}

__global__ void __launch_bounds__(kBlock) kv_residual_cols(VarBase Bs, VarRefs V, Original O) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    const unsigned long long pol = policy_keep();
    ColTerms acc;
    RayTerms ray;
    MC_VARIANT_LINES(j, Bs.n) {
        const int b = __ldg(Bs.cs + j), e = __ldg(Bs.cs + j + 1);
        double s = 0.0, sd = 0.0, sa = 0.0;
        if (live) {
            for (int p = b; p < e; ++p) {
                const double a = __ldg(Bs.cv + p);
                const size_t qi = (size_t)__ldg(Bs.ri + p) * V.Kp + k;
                const double dv = V.dray[qi];
                s = fma(a, ld_keep(V.ya + qi, pol), s);
                sd = fma(a, dv, sd);
                sa = fma(fabs(a), fabs(dv), sa);
            }
            const size_t q = (size_t)j * V.Kp + k;
            acc.add_b(O, (int)j, s, V.xa[q], V.olo[q], V.ohi[q]);
            ray.add_col_b(O, (int)j, sd, sa, V.olo[q], V.ohi[q]);
        }
    }
    const double vmax = lanes_reduce(acc.vmax, sm, OpMax());
    const double dres = lanes_reduce(acc.dres, sm, OpSum());
    const double pobj = lanes_reduce(acc.pobj, sm, OpSum());
    const double dobj = lanes_reduce(acc.dobj, sm, OpSum());
    const double bad = lanes_reduce(acc.bad, sm, OpSum());
    const double rl = lanes_reduce(ray.l, sm, OpSum());
    const double rcs = lanes_reduce(ray.cscale, sm, OpSum());
    const double rci = lanes_reduce(ray.cinf, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) {
        var_partial(V, SLOT_COL_MAX, k)[blockIdx.x] = vmax;
        var_partial(V, SLOT_COL_DRES, k)[blockIdx.x] = dres;
        var_partial(V, SLOT_COL_POBJ, k)[blockIdx.x] = pobj;
        var_partial(V, SLOT_COL_DOBJ, k)[blockIdx.x] = dobj;
        var_partial(V, SLOT_B, k)[blockIdx.x] = bad;
        var_partial(V, SLOT_RAY_L, k)[blockIdx.x] = rl;
        var_partial(V, SLOT_RAY_CSCALE, k)[blockIdx.x] = rcs;
        var_partial(V, SLOT_RAY_CINF, k)[blockIdx.x] = rci;
    }
}

// One block per variant: KKT scalars, termination (optimal, or infeasible by
// the Farkas test), restart and primal weight (pdlp.cpp:229-261).
__global__ void kv_finalize(VarRefs V, double offset, long long span, int final_pass, Controls ctl) {
    __shared__ double scratch[32];
    const int k = blockIdx.x;
    DevState* st = V.st + k;
    if (st->done) return;
    const int nb = V.nb;
    const double row_max = reduce_partials(var_partial(V, SLOT_ROW_MAX, k), nb, scratch, OpMax());
    const double row_dobj = reduce_partials(var_partial(V, SLOT_ROW_DOBJ, k), nb, scratch, OpSum());
    const double bad_r = reduce_partials(var_partial(V, SLOT_NAN, k), nb, scratch, OpSum());
    const double col_max = reduce_partials(var_partial(V, SLOT_COL_MAX, k), nb, scratch, OpMax());
    const double col_dres = reduce_partials(var_partial(V, SLOT_COL_DRES, k), nb, scratch, OpSum());
    const double col_pobj = reduce_partials(var_partial(V, SLOT_COL_POBJ, k), nb, scratch, OpSum());
    const double col_dobj = reduce_partials(var_partial(V, SLOT_COL_DOBJ, k), nb, scratch, OpSum());
    const double bad_c = reduce_partials(var_partial(V, SLOT_B, k), nb, scratch, OpSum());
    const double ray_l = reduce_partials(var_partial(V, SLOT_RAY_L, k), nb, scratch, OpSum());
    const double ray_cs = reduce_partials(var_partial(V, SLOT_RAY_CSCALE, k), nb, scratch, OpSum());
    const double ray_ci = reduce_partials(var_partial(V, SLOT_RAY_CINF, k), nb, scratch, OpSum());
    const double ray_rs = reduce_partials(var_partial(V, SLOT_RAY_RSCALE, k), nb, scratch, OpSum());
    const double ray_ri = reduce_partials(var_partial(V, SLOT_RAY_RINF, k), nb, scratch, OpSum());
    const double ray_u = reduce_partials(var_partial(V, SLOT_RAY_U, k), nb, scratch, OpSum());
    if (threadIdx.x != 0) return;
    const double primal = maxv(row_max, col_max);
    const double dual = sqrt(col_dres) / st->c_scale;
    const double pobj = offset + col_pobj;
    const double dobj = (offset + row_dobj) + col_dobj;
    const double gap = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double score = maxv(maxv(primal, dual), gap);
    const double margin = ray_l - ray_u;
    const bool farkas = ray_ci == 0.0 && ray_ri == 0.0 && margin > 0.0 && margin > 1e-9 * (ray_cs + ray_rs);
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
        st->status = 2;
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

// restart to the average (pdlp.cpp:257-258) of the variants that restart
__global__ void __launch_bounds__(kBlock) kv_restart_copy(VarBase Bs, VarRefs V) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    if (k >= V.K) return;
    const DevState& s = V.st[k];
    if (!s.restart_pending || s.done) return;
    MC_VARIANT_LINES(l, (long long)Bs.n + Bs.m) {
        if (l < Bs.n) {
            const size_t q = (size_t)l * V.Kp + k;
            V.x[q] = V.xa[q];
        } else {
            const size_t q = (size_t)(l - Bs.n) * V.Kp + k;
            V.y[q] = V.ya[q];
        }
    }
}

// the poll flag: done once every variant is
__global__ void kv_poll(VarRefs V) {
    __shared__ int running;
    if (threadIdx.x == 0) running = 0;
    __syncthreads();
    int mine = 0;
    for (int k = threadIdx.x; k < V.K; k += blockDim.x) mine += V.st[k].done ? 0 : 1;
    if (mine) atomicAdd(&running, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        V.global->done = running == 0 ? 1 : 0;
        V.global->active_tiles[0] = running;
    }
}

// ------------------------------------------------------------------ setup
// Variant bounds (given [K][n], original units) into the variant-minor
// arrays: scaled and sentinel forms, the crossed-bound certificate, and the
// start x = proj(given start or 0) (pdlp.cpp:186-191).  Padding lanes get
// zeros, so that gathers over them read finite values.
__global__ void __launch_bounds__(kBlock) kv_setup_cols(VarBase Bs, VarRefs V, const int* __restrict__ perm,
                                                        const double* __restrict__ lo_in,
                                                        const double* __restrict__ hi_in,
                                                        const double* __restrict__ warm_x,
                                                        const int* __restrict__ has_warm_x,
                                                        const double* __restrict__ col_scale) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    const bool real = k < V.K;
    MC_VARIANT_LINES(j, Bs.n) {
        const size_t q = (size_t)j * V.Kp + k;
        if (!real) {
            V.lo[q] = V.hi[q] = V.olo[q] = V.ohi[q] = 0.0;
            V.x[q] = V.xa[q] = V.xb[q] = 0.0;
            V.xdx[2 * q] = V.xdx[2 * q + 1] = 0.0;
            continue;
        }
        const int b = perm[k];  // the caller's variant in slot k
        const size_t g = (size_t)b * Bs.n + j;
        const double s = col_scale[j];
        const double inv = 1.0 / s;
        const double l0 = lo_in[g], h0 = hi_in[g];
        const double ls = isfinite(l0) ? __dmul_rn(l0, inv) : l0;
        const double hs = isfinite(h0) ? __dmul_rn(h0, inv) : h0;
        const double lsent = isinf(ls) ? -kBig : ls;
        const double hsent = isinf(hs) ? kBig : hs;
        V.lo[q] = lsent;
        V.hi[q] = hsent;
        V.olo[q] = isinf(l0) ? -kBig : l0;
        V.ohi[q] = isinf(h0) ? kBig : h0;
        if (l0 > h0) {
            atomicOr(V.flags + k, 1);
            atomicMin(V.cert_idx + k, (int)j);
        }
        const double start = (has_warm_x && has_warm_x[b]) ? __dmul_rn(warm_x[g], inv) : 0.0;
        const double x0 = clampv(start, lsent, hsent);
        V.x[q] = x0;
        V.xa[q] = x0;
        V.xb[q] = x0;
        V.xdx[2 * q] = x0;
        V.xdx[2 * q + 1] = 0.0;
    }
}

// Row-activity certificate per variant (the packed batch's kb_setup_rows
// test on the variant's box) and the dual start.
__global__ void __launch_bounds__(kBlock) kv_setup_rows(VarBase Bs, VarRefs V, const int* __restrict__ perm,
                                                        const double* __restrict__ rlo_in,
                                                        const double* __restrict__ rhi_in,
                                                        const double* __restrict__ row_scale,
                                                        const double* __restrict__ col_scale,
                                                        const double* __restrict__ warm_y,
                                                        const int* __restrict__ has_warm_y) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    const bool real = k < V.K;
    MC_VARIANT_LINES(i, Bs.m) {
        const size_t q = (size_t)i * V.Kp + k;
        if (!real) {
            V.y[q] = V.ya[q] = V.axb[q] = V.y_prev[q] = V.dray[q] = 0.0;
            continue;
        }
        const double s = row_scale[i];
        const double l0 = rlo_in[i], h0 = rhi_in[i];
        double amin = 0.0, amax = 0.0, mag = 0.0;
        for (int p = Bs.rs[i]; p < Bs.rs[i + 1]; ++p) {
            const int j = Bs.ci[p];
            const double a = Bs.rv[p] / (s * col_scale[j]);
            const size_t qj = (size_t)j * V.Kp + k;
            const double lj = V.olo[qj], hj = V.ohi[qj];
            const double t1 = fabs(lj) >= 1e299 ? copysign(INFINITY, lj) * a : a * lj;
            const double t2 = fabs(hj) >= 1e299 ? copysign(INFINITY, hj) * a : a * hj;
            amin += (a > 0) ? t1 : t2;
            amax += (a > 0) ? t2 : t1;
            mag += fabs(a) * maxv(fabs(lj) < 1e299 ? fabs(lj) : 0.0, fabs(hj) < 1e299 ? fabs(hj) : 0.0);
        }
        const double slack =
            1e-9 * (1.0 + mag + maxv(isfinite(l0) ? fabs(l0) : 0.0, isfinite(h0) ? fabs(h0) : 0.0));
        if ((isfinite(l0) && amax < l0 - slack) || (isfinite(h0) && amin > h0 + slack)) {
            atomicOr(V.flags + k, 2);
            atomicMin(V.cert_idx + V.K + k, (int)i);
        }
        const int b = perm[k];
        const double y0 = (has_warm_y && has_warm_y[b]) ? __dmul_rn(warm_y[(size_t)b * Bs.m + i], 1.0 / s) : 0.0;
        V.y[q] = y0;
        V.ya[q] = y0;
        V.axb[q] = 0.0;
        V.y_prev[q] = y0;
        V.dray[q] = 0.0;
    }
}

// every variant starts from the base LP's scalars (pdlp.cpp:153-185): the
// norms, the initial primal weight and eta depend on A, c and the row bounds only
__global__ void kv_setup_state(VarRefs V, const DevState* __restrict__ base) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V.K; k += gridDim.x * blockDim.x) {
        DevState s = *base;
        s.iter = s.avg_count = s.iters_since_restart = s.restarts = s.checks = 0;
        s.restart_pending = 0;
        s.nonfinite = 0;
        s.last_restart_score = 1e300;
        s.primal_infeas = s.dual_infeas = s.gap = 1e300;
        if (V.flags[k]) {
            s.done = 1;
            s.status = 2;
            s.cert = (V.flags[k] & 1) ? MC_CERT_CROSSED_BOUNDS : MC_CERT_ROW_ACTIVITY;
        } else {
            s.done = 0;
            s.status = 1;
            s.cert = MC_CERT_NONE;
        }
        V.st[k] = s;
    }
}

// unscaled averages of every variant into [K][n] and [K][m] staging
__global__ void __launch_bounds__(kBlock) kv_unscale_out(VarBase Bs, VarRefs V, const double* __restrict__ col_scale,
                                                         const double* __restrict__ row_scale, double* __restrict__ xo,
                                                         double* __restrict__ yo) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    if (k >= V.K) return;
    // a variant proven infeasible by a dual ray returns the ray as its dual
    const bool ray = V.st[k].status == 2 && V.st[k].cert == MC_CERT_DUAL_RAY;
    const double* yv = ray ? V.dray : V.ya;
    MC_VARIANT_LINES(l, (long long)Bs.n + Bs.m) {
        if (l < Bs.n) {
            xo[(size_t)k * Bs.n + l] = __dmul_rn(V.xa[(size_t)l * V.Kp + k], col_scale[l]);
        } else {
            const long long i = l - Bs.n;
            yo[(size_t)k * Bs.m + i] = __dmul_rn(yv[(size_t)i * V.Kp + k], row_scale[i]);
        }
    }
}

// ------------------------------------------------------------ the engine
struct EngineVariants {
    VarBase Bs;
    VarRefs V;
    Original O;
    dim3 grid;
    int shape_class(const DevState&) const { return 0; }
    void use_class(int) const {}

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) kv_primal<true><<<grid, kBlock, 0, s>>>(Bs, V, k);
        else kv_primal<false><<<grid, kBlock, 0, s>>>(Bs, V, k);
        ctx.end_launch();
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kv_dual_probe<<<grid, kBlock, 0, s>>>(Bs, V);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            kv_step_size<<<V.K, 256, 0, s>>>(V, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kv_dual_apply<<<grid, kBlock, 0, s>>>(Bs, V, k);
            ctx.end_launch();
        } else {
            ctx.begin_launch(MC_KERNEL_DUAL);
            kv_dual<<<grid, kBlock, 0, s>>>(Bs, V, k);
            ctx.end_launch();
        }
        return ctx.launch_check("variant iteration");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf&) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kv_residual_rows<<<grid, kBlock, 0, s>>>(Bs, V, O);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kv_residual_cols<<<grid, kBlock, 0, s>>>(Bs, V, O);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kv_finalize<<<V.K, 256, 0, s>>>(V, O.offset, span, final_pass, ctl);
        ctx.end_launch();
        if (!final_pass) {
            ctx.begin_launch(MC_KERNEL_OTHER);
            kv_restart_copy<<<grid, kBlock, 0, s>>>(Bs, V);
            ctx.end_launch();
        }
        ctx.begin_launch(MC_KERNEL_OTHER);
        kv_poll<<<1, 1024, 0, s>>>(V);
        ctx.end_launch();
        return ctx.launch_check("variant check");
    }
};

// ----------------------------------------------------- the FP32 form
// The mixed-precision form of mixed.cuh per variant: each variant's iterate
// is an FP64 base plus an FP32 correction, x = xh + dx, y = yh + dy; FP32 PDHG
// runs on the correction LP (FP32 matrix, FP32 variant-minor vectors); the
// residual pass, gap, restart test and primal weight are FP64 on xh + dx_avg
// with the FP64 matrix; at every restart a variant's base moves to its average
// and its correction LP is rebuilt from the residual pass's FP64 products.
struct VarMixed {
    const int* cs;          // the base's CSC / CSR structure (shared with the FP64 data)
    const int* ri;
    const float* cv;        // FP32 matrix values
    const int* rs;
    const int* ci;
    const float* rv;
    const float* col_norm;  // FP32 norms
    const float* row_norm;
    const double* c64;      // scaled c, FP64
    const double* blo64;    // scaled row bounds, sentinel form, FP64
    const double* bhi64;
    double* xh;             // [n Kp] FP64 bases
    double* yh;             // [m Kp]
    double* axf;            // [m Kp] A (xh + dx_avg) from the residual pass
    double* atyf;           // [n Kp] A^T (yh + dy_avg)
    float* x;               // [n Kp] dx
    float* xb;              // [n Kp] dx-bar
    float* xa;              // [n Kp] dx average
    float* xdx;             // [2 n Kp] (dx-bar, d dx) pairs
    float* g;               // [n Kp] float(c + A^T yh)
    float* lo;              // [n Kp] float(lo - xh), +-inf when unbounded
    float* hi;
    float* y;               // [m Kp] dy
    float* ya;              // [m Kp] dy average
    float* axb;             // [m Kp] A dx-bar of a step-size iteration
    float* yb;              // [m Kp] float(yh)
    float* rlo;             // [m Kp] float(A xh - b_lo), +inf when unbounded
    float* rhi;             // [m Kp] float(A xh - b_hi), -inf when unbounded
};

__device__ __forceinline__ float variant_dot_f(const int* __restrict__ start, const int* __restrict__ idx,
                                               const float* __restrict__ val, const float* __restrict__ v, int Kp,
                                               long long l, int k, bool live, unsigned long long pol) {
    const int b = __ldg(start + l), e = __ldg(start + l + 1);
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int p = b;
    for (; p + 4 <= e; p += 4) {
        const int i0 = __ldg(idx + p), i1 = __ldg(idx + p + 1), i2 = __ldg(idx + p + 2), i3 = __ldg(idx + p + 3);
        const float a0 = __ldg(val + p), a1 = __ldg(val + p + 1), a2 = __ldg(val + p + 2), a3 = __ldg(val + p + 3);
        if (live) {
            s0 = fmaf(a0, ld_keep(v + (size_t)i0 * Kp + k, pol), s0);
            s1 = fmaf(a1, ld_keep(v + (size_t)i1 * Kp + k, pol), s1);
            s2 = fmaf(a2, ld_keep(v + (size_t)i2 * Kp + k, pol), s2);
            s3 = fmaf(a3, ld_keep(v + (size_t)i3 * Kp + k, pol), s3);
        }
    }
    for (; p < e; ++p)
        if (live) s0 = fmaf(__ldg(val + p), ld_keep(v + (size_t)__ldg(idx + p) * Kp + k, pol), s0);
    return (s0 + s1) + (s2 + s3);
}

template <bool STEP>
__global__ void __launch_bounds__(kBlock) kvm_primal(int n, VarRefs V, VarMixed M, int kk) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    float step = 0.f, cnt = 1.f;
    if (live) {
        const DevState& s = V.st[k];
        step = (float)(s.eta / s.omega);
        cnt = (float)(double)(s.avg_count + kk + 1);
    }
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    MC_VARIANT_LINES(j, n) {
        const float aty = variant_dot_f(M.cs, M.ri, M.cv, M.y, V.Kp, j, k, live, pol);
        if (live) {
            const size_t q = (size_t)j * V.Kp + k;
            const float cn = __ldg(M.col_norm + j);
            const float g = __fadd_rn(ld_stream(M.g + q), aty);
            const float tau = __fdiv_rn(step, cn);
            const float xo = ld_stream(M.x + q);
            const float xp = clampv(__fsub_rn(xo, __fmul_rn(tau, g)), ld_stream(M.lo + q), ld_stream(M.hi + q));
            const float d = __fsub_rn(xp, xo);
            const float xbar = __fsub_rn(__fmul_rn(2.f, xp), xo);
            if (STEP) {
                st_keep2(M.xdx + 2 * q, xbar, d, pol);
                acc += __dmul_rn(__dmul_rn((double)cn, (double)d), (double)d);
            } else {
                st_keep(M.xb + q, xbar, pol);
            }
            st_stream(M.x + q, xp);
            const float xa = ld_stream(M.xa + q);
            st_stream(M.xa + q, __fadd_rn(xa, __fdiv_rn(__fsub_rn(xp, xa), cnt)));
        }
    }
    if (STEP) {
        acc = lanes_reduce(acc, sm, OpSum());
        if ((threadIdx.x >> 5) == 0 && k < V.K) var_partial(V, SLOT_DX, k)[blockIdx.x] = acc;
    }
}

// the dual step on the correction (dual_update_mx of mixed.cuh, per variant)
__device__ __forceinline__ void variant_dual_update_mx(const VarRefs& V, const VarMixed& M, long long i, int k,
                                                       float ax, float sg, float cnt, unsigned long long pol) {
    const size_t q = (size_t)i * V.Kp + k;
    const float sigma = __fdiv_rn(sg, __ldg(M.row_norm + i));
    const float dy = ld_stream(M.y + q), yb = ld_stream(M.yb + q);
    const float rl = ld_stream(M.rlo + q), rh = ld_stream(M.rhi + q);
    const float base = __fdiv_rn(__fadd_rn(yb, dy), sigma);
    float dyn;
    if (__fadd_rn(base, __fadd_rn(rl, ax)) < 0.f) dyn = __fadd_rn(dy, __fmul_rn(sigma, __fadd_rn(rl, ax)));
    else if (__fadd_rn(base, __fadd_rn(rh, ax)) > 0.f) dyn = __fadd_rn(dy, __fmul_rn(sigma, __fadd_rn(rh, ax)));
    else dyn = -yb;
    st_keep(M.y + q, dyn, pol);
    const float dya = ld_stream(M.ya + q);
    st_stream(M.ya + q, __fadd_rn(dya, __fdiv_rn(__fsub_rn(dyn, dya), cnt)));
}

__global__ void __launch_bounds__(kBlock) kvm_dual(int m, VarRefs V, VarMixed M, int kk) {
    MC_VARIANT_LANE(V, k, live);
    float sg = 0.f, cnt = 1.f;
    if (live) {
        const DevState& s = V.st[k];
        sg = (float)(s.eta * s.omega);
        cnt = (float)(double)(s.avg_count + kk + 1);
    }
    const unsigned long long pol = policy_keep();
    MC_VARIANT_LINES(i, m) {
        const float ax = variant_dot_f(M.rs, M.ci, M.rv, M.xb, V.Kp, i, k, live, pol);
        if (live) variant_dual_update_mx(V, M, i, k, ax, sg, cnt, pol);
    }
}

__global__ void __launch_bounds__(kBlock) kvm_dual_probe(int m, VarRefs V, VarMixed M) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    const unsigned long long pol = policy_keep();
    double acc = 0.0;
    MC_VARIANT_LINES(i, m) {
        const int b = __ldg(M.rs + i), e = __ldg(M.rs + i + 1);
        float sv0 = 0.f, sw0 = 0.f, sv1 = 0.f, sw1 = 0.f;
        int p = b;
        for (; p + 2 <= e; p += 2) {
            const int j0 = __ldg(M.ci + p), j1 = __ldg(M.ci + p + 1);
            const float a0 = __ldg(M.rv + p), a1 = __ldg(M.rv + p + 1);
            if (live) {
                float v0, w0, v1, w1;
                ld_keep2(M.xdx + 2 * ((size_t)j0 * V.Kp + k), pol, v0, w0);
                ld_keep2(M.xdx + 2 * ((size_t)j1 * V.Kp + k), pol, v1, w1);
                sv0 = fmaf(a0, v0, sv0);
                sw0 = fmaf(a0, w0, sw0);
                sv1 = fmaf(a1, v1, sv1);
                sw1 = fmaf(a1, w1, sw1);
            }
        }
        if (p < e && live) {
            float v0, w0;
            ld_keep2(M.xdx + 2 * ((size_t)__ldg(M.ci + p) * V.Kp + k), pol, v0, w0);
            const float a0 = __ldg(M.rv + p);
            sv0 = fmaf(a0, v0, sv0);
            sw0 = fmaf(a0, w0, sw0);
        }
        if (live) {
            M.axb[(size_t)i * V.Kp + k] = sv0 + sv1;
            const double adx = (double)(sw0 + sw1);
            acc += __ddiv_rn(__dmul_rn(adx, adx), (double)__ldg(M.row_norm + i));
        }
    }
    acc = lanes_reduce(acc, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) var_partial(V, SLOT_ADX, k)[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kBlock) kvm_dual_apply(int m, VarRefs V, VarMixed M, int kk) {
    MC_VARIANT_LANE(V, k, live);
    if (!live) return;  // no barrier follows
    const DevState& s = V.st[k];
    const float sg = (float)(s.eta * s.omega);
    const float cnt = (float)(double)(s.avg_count + kk + 1);
    const unsigned long long pol = policy_keep();
    MC_VARIANT_LINES(i, m) variant_dual_update_mx(V, M, i, k, M.axb[(size_t)i * V.Kp + k], sg, cnt, pol);
}

// FP64 residual pass on xh + dx_avg, yh + dy_avg (FP64 matrix of the base),
// keeping A x and A^T y of that point for the recentring; Farkas terms.
__global__ void __launch_bounds__(kBlock) kvm_residual_rows(VarBase Bs, VarRefs V, VarMixed M, Original O) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    RowTerms acc;
    RayTerms ray;
    MC_VARIANT_LINES(i, Bs.m) {
        double s = 0.0;
        if (live) {
            for (int p = __ldg(Bs.rs + i); p < __ldg(Bs.rs + i + 1); ++p) {
                const size_t qj = (size_t)__ldg(Bs.ci + p) * V.Kp + k;
                s = fma(__ldg(Bs.rv + p), M.xh[qj] + (double)M.xa[qj], s);
            }
            const size_t q = (size_t)i * V.Kp + k;
            M.axf[q] = s;
            const double yv = M.yh[q] + (double)M.ya[q];
            acc.add(O, (int)i, s, yv);
            const double d = RayTerms::candidate(O, (int)i, yv, V.y_prev + q);
            V.dray[q] = d;
            ray.add_row(O, (int)i, d);
        }
    }
    const double vmax = lanes_reduce(acc.vmax, sm, OpMax());
    const double dsum = lanes_reduce(acc.dsum, sm, OpSum());
    const double bad = lanes_reduce(acc.bad, sm, OpSum());
    const double ru = lanes_reduce(ray.u, sm, OpSum());
    const double rsc = lanes_reduce(ray.rscale, sm, OpSum());
    const double rinf = lanes_reduce(ray.rinf, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) {
        var_partial(V, SLOT_ROW_MAX, k)[blockIdx.x] = vmax;
        var_partial(V, SLOT_ROW_DOBJ, k)[blockIdx.x] = dsum;
        var_partial(V, SLOT_NAN, k)[blockIdx.x] = bad;
        var_partial(V, SLOT_RAY_U, k)[blockIdx.x] = ru;
        var_partial(V, SLOT_RAY_RSCALE, k)[blockIdx.x] = rsc;
        var_partial(V, SLOT_RAY_RINF, k)[blockIdx.x] = rinf;
    }
}

__global__ void __launch_bounds__(kBlock) kvm_residual_cols(VarBase Bs, VarRefs V, VarMixed M, Original O) {
    __shared__ double sm[kVarWarps][33];
    MC_VARIANT_LANE(V, k, live);
    ColTerms acc;
    RayTerms ray;
    MC_VARIANT_LINES(j, Bs.n) {
        double s = 0.0, sd = 0.0, sa = 0.0;
        if (live) {
            for (int p = __ldg(Bs.cs + j); p < __ldg(Bs.cs + j + 1); ++p) {
                const double a = __ldg(Bs.cv + p);
                const size_t qi = (size_t)__ldg(Bs.ri + p) * V.Kp + k;
                const double dv = V.dray[qi];
                s = fma(a, M.yh[qi] + (double)M.ya[qi], s);
                sd = fma(a, dv, sd);
                sa = fma(fabs(a), fabs(dv), sa);
            }
            const size_t q = (size_t)j * V.Kp + k;
            M.atyf[q] = s;
            acc.add_b(O, (int)j, s, M.xh[q] + (double)M.xa[q], V.olo[q], V.ohi[q]);
            ray.add_col_b(O, (int)j, sd, sa, V.olo[q], V.ohi[q]);
        }
    }
    const double vmax = lanes_reduce(acc.vmax, sm, OpMax());
    const double dres = lanes_reduce(acc.dres, sm, OpSum());
    const double pobj = lanes_reduce(acc.pobj, sm, OpSum());
    const double dobj = lanes_reduce(acc.dobj, sm, OpSum());
    const double bad = lanes_reduce(acc.bad, sm, OpSum());
    const double rl = lanes_reduce(ray.l, sm, OpSum());
    const double rcs = lanes_reduce(ray.cscale, sm, OpSum());
    const double rci = lanes_reduce(ray.cinf, sm, OpSum());
    if ((threadIdx.x >> 5) == 0 && k < V.K) {
        var_partial(V, SLOT_COL_MAX, k)[blockIdx.x] = vmax;
        var_partial(V, SLOT_COL_DRES, k)[blockIdx.x] = dres;
        var_partial(V, SLOT_COL_POBJ, k)[blockIdx.x] = pobj;
        var_partial(V, SLOT_COL_DOBJ, k)[blockIdx.x] = dobj;
        var_partial(V, SLOT_B, k)[blockIdx.x] = bad;
        var_partial(V, SLOT_RAY_L, k)[blockIdx.x] = rl;
        var_partial(V, SLOT_RAY_CSCALE, k)[blockIdx.x] = rcs;
        var_partial(V, SLOT_RAY_CINF, k)[blockIdx.x] = rci;
    }
}

// Restart of a variant to its average: its base moves there and its
// correction LP is rebuilt from the residual pass's FP64 products
// (k_recenter_mx per variant).  `force` rebuilds every running variant.
__global__ void __launch_bounds__(kBlock) kvm_recenter(int m, int n, VarRefs V, VarMixed M, int force) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    if (k >= V.K) return;
    const DevState& s = V.st[k];
    if (s.done || (!force && !s.restart_pending)) return;
    const float inf = __int_as_float(0x7f800000);
    MC_VARIANT_LINES(l, (long long)n + m) {
        if (l < n) {
            const size_t q = (size_t)l * V.Kp + k;
            const double xh = M.xh[q] + (double)M.xa[q];
            M.xh[q] = xh;
            M.x[q] = 0.f;
            M.xa[q] = 0.f;
            M.g[q] = (float)(M.c64[l] + M.atyf[q]);
            const double lo = V.lo[q], hi = V.hi[q];
            M.lo[q] = (lo <= -1e299) ? -inf : (float)(lo - xh);
            M.hi[q] = (hi >= 1e299) ? inf : (float)(hi - xh);
        } else {
            const long long i = l - n;
            const size_t q = (size_t)i * V.Kp + k;
            const double yh = M.yh[q] + (double)M.ya[q];
            M.yh[q] = yh;
            M.y[q] = 0.f;
            M.ya[q] = 0.f;
            M.yb[q] = (float)yh;
            const double ax = M.axf[q], lo = M.blo64[i], hi = M.bhi64[i];
            M.rlo[q] = (lo <= -1e299) ? inf : (float)(ax - lo);
            M.rhi[q] = (hi >= 1e299) ? -inf : (float)(ax - hi);
        }
    }
}

// unscaled outputs of the FP32 form: x = (xh + dx_avg) D_C, y = (yh + dy_avg) D_R
// (the ray for a variant proven infeasible by one)
__global__ void __launch_bounds__(kBlock) kvm_unscale_out(int m, int n, VarRefs V, VarMixed M,
                                                          const double* __restrict__ col_scale,
                                                          const double* __restrict__ row_scale,
                                                          double* __restrict__ xo, double* __restrict__ yo) {
    const int k = blockIdx.y * 32 + (threadIdx.x & 31);
    if (k >= V.K) return;
    const bool ray = V.st[k].status == 2 && V.st[k].cert == MC_CERT_DUAL_RAY;
    MC_VARIANT_LINES(l, (long long)n + m) {
        if (l < n) {
            const size_t q = (size_t)l * V.Kp + k;
            xo[(size_t)k * n + l] = __dmul_rn(M.xh[q] + (double)M.xa[q], col_scale[l]);
        } else {
            const long long i = l - n;
            const size_t q = (size_t)i * V.Kp + k;
            const double yv = ray ? V.dray[q] : M.yh[q] + (double)M.ya[q];
            yo[(size_t)k * m + i] = __dmul_rn(yv, row_scale[i]);
        }
    }
}

struct EngineVariantsMixed {
    VarBase Bs;
    VarRefs V;
    VarMixed M;
    Original O;
    dim3 grid;
    int shape_class(const DevState&) const { return 0; }
    void use_class(int) const {}

    int iteration(Ctx& ctx, int k, bool step, const Controls& ctl) const {
        cudaStream_t s = ctx.stream;
        ctx.begin_launch(MC_KERNEL_PRIMAL);
        if (step) kvm_primal<true><<<grid, kBlock, 0, s>>>(Bs.n, V, M, k);
        else kvm_primal<false><<<grid, kBlock, 0, s>>>(Bs.n, V, M, k);
        ctx.end_launch();
        if (step) {
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kvm_dual_probe<<<grid, kBlock, 0, s>>>(Bs.m, V, M);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_OTHER);
            kv_step_size<<<V.K, 256, 0, s>>>(V, ctl);
            ctx.end_launch();
            ctx.begin_launch(MC_KERNEL_DUAL_STEP);
            kvm_dual_apply<<<grid, kBlock, 0, s>>>(Bs.m, V, M, k);
            ctx.end_launch();
        } else {
            ctx.begin_launch(MC_KERNEL_DUAL);
            kvm_dual<<<grid, kBlock, 0, s>>>(Bs.m, V, M, k);
            ctx.end_launch();
        }
        return ctx.launch_check("variant iteration (FP32)");
    }

    int residual_pass(Ctx& ctx) const {
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kvm_residual_rows<<<grid, kBlock, 0, ctx.stream>>>(Bs, V, M, O);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kvm_residual_cols<<<grid, kBlock, 0, ctx.stream>>>(Bs, V, M, O);
        ctx.end_launch();
        return ctx.launch_check("variant residual (FP32)");
    }

    int recenter(Ctx& ctx, int force) const {
        ctx.begin_launch(MC_KERNEL_OTHER);
        kvm_recenter<<<grid, kBlock, 0, ctx.stream>>>(Bs.m, Bs.n, V, M, force);
        ctx.end_launch();
        return ctx.launch_check("variant recenter");
    }

    int check(Ctx& ctx, long long span, int final_pass, const Controls& ctl, const TraceBuf&) const {
        TRY(residual_pass(ctx));
        ctx.begin_launch(MC_KERNEL_RESIDUAL);
        kv_finalize<<<V.K, 256, 0, ctx.stream>>>(V, O.offset, span, final_pass, ctl);
        ctx.end_launch();
        if (!final_pass) TRY(recenter(ctx, 0));
        ctx.begin_launch(MC_KERNEL_OTHER);
        kv_poll<<<1, 1024, 0, ctx.stream>>>(V);
        ctx.end_launch();
        return ctx.launch_check("variant check (FP32)");
    }
};

// Host driver: the base LP's setup as a single solve's (upload, validation,
// transpose, Ruiz, norms), then the variants' bounds, starts and
// certificates, the PDHG loop in chunk graphs, and per-variant outputs.
int solve_variants(Ctx& ctx, const mc_lp* base, int count, const double* const* var_lower,
                   const double* const* var_upper, const mc_pdlp_options* o, const double* const* x0,
                   const double* const* y0, double* const* x_out, double* const* y_out, mc_pdlp_result* results) {
    ctx.drop_session();  // reuses the arena
    const double t_begin = now_ms();
    if (!base || count <= 0 || !results) return set_error(MC_ERR_INVALID_ARGUMENT, "no variants");
    TRY(validate_options(o));
    TRY(validate_lp(base));
    const bool mixed = o->precision == MC_PRECISION_FP32_REFINE;
    const int m = base->num_rows, n = base->num_cols;
    const long long nnz = base->nnz;
    for (int b = 0; b < count; ++b) {
        std::memset(&results[b], 0, sizeof(mc_pdlp_result));
        std::snprintf(results[b].backend_actually_used, sizeof results[b].backend_actually_used, "cuda");
        results[b].tolerance = o->primal_tolerance;
        results[b].certificate_index = -1;
    }
    if (m == 0 || n == 0) {  // pdlp.cpp:144-149, for every variant
        for (int b = 0; b < count; ++b) {
            results[b].status = MC_PDLP_OPTIMAL;
            fill_message(&results[b], "trivial");
            results[b].total_ms = now_ms() - t_begin;
        }
        return MC_OK;
    }
    const int Kp = (count + 31) / 32 * 32;
    const int groups = Kp / 32;
    if (groups > 65535) return set_error(MC_ERR_RESOURCE_LIMIT, "too many variants (%d)", count);
    cudaStream_t s = ctx.stream;
    for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
        ctx.launches[q] = 0;
        ctx.kernel_ms[q] = 0.0;
    }
    ctx.profiling = o->profile_kernels != 0;
    ctx.pending.clear();
    ctx.prof_used = 0;
    ctx.release_graphs();

    // grid: (blocks per variant group, variant groups), about two waves of resident blocks
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kv_residual_cols, kBlock, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const long long lines = std::max<long long>(n, m);
    long long nbx = std::max<long long>(1, (long long)ctx.sm_count * per_sm * 2 / groups);
    nbx = std::min<long long>(nbx, (lines + kVarWarps - 1) / kVarWarps);
    nbx = std::max<long long>(1, std::min<long long>(nbx, kMaxPartials));

    // ---- arena
    const bool dev_in = base->memory == MC_MEMORY_DEVICE;
    bool any_wx = false, any_wy = false;
    for (int b = 0; b < count; ++b) {
        any_wx = any_wx || (x0 && x0[b]);
        any_wy = any_wy || (y0 && y0[b]);
    }
    Layout L;
    const size_t o_cs = L.add<int>(n + 1), o_ri = L.add<int>(nnz + 16), o_cv = L.add<double>(nnz + 16);
    const size_t o_rs = L.add<int>(m + 1), o_ci = L.add<int>(nnz + 16), o_rv = L.add<double>(nnz + 16);
    const size_t o_cursor = L.add<int>(m), o_long = L.add<int>(m), o_counters = L.add<int>(4);
    const size_t o_scan = L.add<int>((m + 1) / kScanTile + 4096);
    size_t o_n[12], o_m[9];
    for (auto& v : o_n) v = L.add<double>(n);
    for (auto& v : o_m) v = L.add<double>(m);
    const size_t o_part1 = L.add<double>((long long)NUM_SLOTS * kMaxPartials);
    const size_t o_state = L.add<DevState>(count + 2);
    const long long nk = (long long)n * Kp, mk = (long long)m * Kp;
    size_t o_vn[7], o_vm[5];
    for (auto& v : o_vn) v = L.add<double>(nk);
    const size_t o_vxdx = L.add<double>(2 * nk);
    for (auto& v : o_vm) v = L.add<double>(mk);
    const size_t o_vpart = L.add<double>((long long)NUM_SLOTS * Kp * nbx);
    const size_t o_flags = L.add<int>(count), o_cert = L.add<int>(2LL * count);
    const size_t o_lo_in = L.add<double>((long long)count * n), o_hi_in = L.add<double>((long long)count * n);
    const size_t o_wx = any_wx ? L.add<double>((long long)count * n) : 0;
    const size_t o_wy = any_wy ? L.add<double>((long long)count * m) : 0;
    const size_t o_hw = L.add<int>(2LL * count);
    const size_t o_perm = L.add<int>(count);
    const size_t o_xo = L.add<double>((long long)count * n), o_yo = L.add<double>((long long)count * m);
    // FP32 form: FP32 matrix copies and norms, FP32 variant-minor correction data
    size_t o_f_cv = 0, o_f_rv = 0, o_f_cn = 0, o_f_rn = 0, o_fn[7] = {}, o_fxdx = 0, o_fm[6] = {};
    if (mixed) {
        o_f_cv = L.add<float>(nnz + 16);
        o_f_rv = L.add<float>(nnz + 16);
        o_f_cn = L.add<float>(n);
        o_f_rn = L.add<float>(m);
        for (auto& v : o_fn) v = L.add<float>(nk);
        o_fxdx = L.add<float>(2 * nk);
        for (auto& v : o_fm) v = L.add<float>(mk);
    }
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
    double* base_lo_in = static_cast<double*>(at(o_n[1]));  // base variable bounds (base setup only)
    double* base_hi_in = static_cast<double*>(at(o_n[2]));
    double* c = static_cast<double*>(at(o_n[3]));
    double* lo_b = static_cast<double*>(at(o_n[4]));
    double* hi_b = static_cast<double*>(at(o_n[5]));
    double* c_orig = static_cast<double*>(at(o_n[6]));
    double* lo_orig = static_cast<double*>(at(o_n[7]));
    double* hi_orig = static_cast<double*>(at(o_n[8]));
    double* col_norm = static_cast<double*>(at(o_n[9]));
    double* col_scale = static_cast<double*>(at(o_n[10]));
    double* x_scratch = static_cast<double*>(at(o_n[11]));
    double* rlo_in = static_cast<double*>(at(o_m[0]));
    double* rhi_in = static_cast<double*>(at(o_m[1]));
    double* blo = static_cast<double*>(at(o_m[2]));
    double* bhi = static_cast<double*>(at(o_m[3]));
    double* blo_orig = static_cast<double*>(at(o_m[4]));
    double* bhi_orig = static_cast<double*>(at(o_m[5]));
    double* row_norm = static_cast<double*>(at(o_m[6]));
    double* row_scale = static_cast<double*>(at(o_m[7]));
    double* y_scratch = static_cast<double*>(at(o_m[8]));
    double* part1 = static_cast<double*>(at(o_part1));
    DevState* st = static_cast<DevState*>(at(o_state));  // [0] base, [1] poll, [2..] variants
    int* has_warm = static_cast<int*>(at(o_hw));

    // ---- uploads and validation of the base
    CU(cudaEventRecord(ctx.ev_a, s));
    const cudaMemcpyKind in_kind = dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CU(cudaMemcpyAsync(cs, base->col_start, sizeof(int) * (size_t)(n + 1), in_kind, s));
    if (nnz) {
        CU(cudaMemcpyAsync(ri, base->row_index, sizeof(int) * (size_t)nnz, in_kind, s));
        CU(cudaMemcpyAsync(cv, base->value, sizeof(double) * (size_t)nnz, in_kind, s));
    }
    CU(cudaMemsetAsync(ri + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(cv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemsetAsync(ci + nnz, 0, sizeof(int) * 16, s));
    CU(cudaMemsetAsync(rv + nnz, 0, sizeof(double) * 16, s));
    CU(cudaMemcpyAsync(obj_in, base->objective, sizeof(double) * n, in_kind, s));
    CU(cudaMemcpyAsync(base_lo_in, base->var_lower, sizeof(double) * n, in_kind, s));
    CU(cudaMemcpyAsync(base_hi_in, base->var_upper, sizeof(double) * n, in_kind, s));
    CU(cudaMemcpyAsync(rlo_in, base->row_lower, sizeof(double) * m, in_kind, s));
    CU(cudaMemcpyAsync(rhi_in, base->row_upper, sizeof(double) * m, in_kind, s));
    double* lo_in = static_cast<double*>(at(o_lo_in));
    double* hi_in = static_cast<double*>(at(o_hi_in));
    double* wx = any_wx ? static_cast<double*>(at(o_wx)) : nullptr;
    double* wy = any_wy ? static_cast<double*>(at(o_wy)) : nullptr;
    std::vector<int> hw(2 * (size_t)count, 0);
    for (int b = 0; b < count; ++b) {
        const double* lb = (var_lower && var_lower[b]) ? var_lower[b] : base->var_lower;
        const double* ub = (var_upper && var_upper[b]) ? var_upper[b] : base->var_upper;
        CU(cudaMemcpyAsync(lo_in + (size_t)b * n, lb, sizeof(double) * n, cudaMemcpyDefault, s));
        CU(cudaMemcpyAsync(hi_in + (size_t)b * n, ub, sizeof(double) * n, cudaMemcpyDefault, s));
        if (x0 && x0[b]) {
            hw[b] = 1;
            CU(cudaMemcpyAsync(wx + (size_t)b * n, x0[b], sizeof(double) * n, cudaMemcpyDefault, s));
        }
        if (y0 && y0[b]) {
            hw[count + b] = 1;
            CU(cudaMemcpyAsync(wy + (size_t)b * m, y0[b], sizeof(double) * m, cudaMemcpyDefault, s));
        }
    }
    CU(cudaMemcpyAsync(has_warm, hw.data(), sizeof(int) * hw.size(), cudaMemcpyHostToDevice, s));
    CU(cudaEventRecord(ctx.ev_b, s));
    int* counters = static_cast<int*>(at(o_counters));
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, cs, ri, cv, counters + 2);
    ctx.end_launch();
    int bad = 0;
    CU(cudaMemcpyAsync(&bad, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.drain_profile());
    if (bad) return set_error(MC_ERR_INVALID_ARGUMENT, "invalid CSC matrix in the base LP (flags %d)", bad);

    // ---- the base LP's setup (shared by every variant)
    CU(cudaMemsetAsync(st, 0, sizeof(DevState) * (count + 2), s));
    TRY(build_csr(ctx, m, n, nnz, cs, ri, cv, rs, ci, rv, static_cast<int*>(at(o_cursor)),
                  static_cast<int*>(at(o_long)), counters, static_cast<int*>(at(o_scan))));
    TRY(ruiz(ctx, m, n, nnz, cs, ri, cv, rs, ci, rv, row_scale, col_scale, y_scratch, x_scratch, part1, st,
             o->ruiz_scaling ? o->ruiz_iterations : 0));
    const double obj_sign = (base->objective_sense == MC_MAXIMIZE) ? -1.0 : 1.0;
    const int nbc = blocks_for(ctx, n, kBlock), nbr = blocks_for(ctx, m, kBlock);
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_setup_cols<<<nbc, kBlock, 0, s>>>(n, cs, cv, obj_in, base_lo_in, base_hi_in, col_scale, nullptr, obj_sign, c,
                                        lo_b, hi_b, c_orig, lo_orig, hi_orig, col_norm, x_scratch, x_scratch, part1);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_setup_rows<<<nbr, kBlock, 0, s>>>(m, rs, rv, rlo_in, rhi_in, row_scale, nullptr, blo, bhi, blo_orig, bhi_orig,
                                        row_norm, y_scratch, y_scratch, part1);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    k_setup_scalars<<<1, 1024, 0, s>>>(part1, nbc, nbr, o->initial_primal_weight, o->step_size_reduction, st);
    ctx.end_launch();

    // ---- the variants
    VarBase Bs{m, n, cs, ri, cv, rs, ci, rv, c, col_norm, row_norm, blo, bhi};
    VarRefs V;
    V.K = count;
    V.Kp = Kp;
    V.nb = (int)nbx;
    V.st = st + 2;
    V.global = st + 1;
    V.lo = static_cast<double*>(at(o_vn[0]));
    V.hi = static_cast<double*>(at(o_vn[1]));
    V.olo = static_cast<double*>(at(o_vn[2]));
    V.ohi = static_cast<double*>(at(o_vn[3]));
    V.x = static_cast<double*>(at(o_vn[4]));
    V.xb = static_cast<double*>(at(o_vn[5]));
    V.xa = static_cast<double*>(at(o_vn[6]));
    V.xdx = static_cast<double*>(at(o_vxdx));
    V.y = static_cast<double*>(at(o_vm[0]));
    V.ya = static_cast<double*>(at(o_vm[1]));
    V.axb = static_cast<double*>(at(o_vm[2]));
    V.y_prev = static_cast<double*>(at(o_vm[3]));
    V.dray = static_cast<double*>(at(o_vm[4]));
    V.partials = static_cast<double*>(at(o_vpart));
    V.flags = static_cast<int*>(at(o_flags));
    V.cert_idx = static_cast<int*>(at(o_cert));
    CU(cudaMemsetAsync(V.partials, 0, sizeof(double) * (size_t)NUM_SLOTS * Kp * nbx, s));
    const dim3 grid((unsigned)nbx, (unsigned)groups);
    // Slots: variant b of the caller sits in slot k with perm[k] = b.  The
    // variants certified infeasible at setup go last, so that the groups of
    // 32 slots that hold only finished variants leave every kernel at once;
    // the certificates are found with the identity order first.
    int* perm_dev = static_cast<int*>(at(o_perm));
    std::vector<int> perm(count);
    for (int b = 0; b < count; ++b) perm[b] = b;
    auto setup_slots = [&]() -> int {
        CU(cudaMemcpyAsync(perm_dev, perm.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
        CU(cudaMemsetAsync(V.flags, 0, sizeof(int) * count, s));
        CU(cudaMemsetAsync(V.cert_idx, 0x7f, sizeof(int) * 2 * (size_t)count, s));  // "none" above any index
        ctx.begin_launch(MC_KERNEL_SETUP);
        kv_setup_cols<<<grid, kBlock, 0, s>>>(Bs, V, perm_dev, lo_in, hi_in, wx, any_wx ? has_warm : nullptr,
                                              col_scale);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        kv_setup_rows<<<grid, kBlock, 0, s>>>(Bs, V, perm_dev, rlo_in, rhi_in, row_scale, col_scale, wy,
                                              any_wy ? has_warm + count : nullptr);
        ctx.end_launch();
        return ctx.launch_check("variant slots");
    };
    TRY(setup_slots());
    {
        std::vector<int> hflags(count);
        CU(cudaMemcpyAsync(hflags.data(), V.flags, sizeof(int) * count, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        TRY(ctx.drain_profile());
        std::vector<int> order;
        order.reserve(count);
        for (int b = 0; b < count; ++b)
            if (!hflags[b]) order.push_back(b);
        for (int b = 0; b < count; ++b)
            if (hflags[b]) order.push_back(b);
        if (order != perm) {
            perm = order;
            TRY(setup_slots());
        }
    }
    ctx.begin_launch(MC_KERNEL_SETUP);
    kv_setup_state<<<(count + 255) / 256, 256, 0, s>>>(V, st);
    ctx.end_launch();
    ctx.begin_launch(MC_KERNEL_SETUP);
    kv_poll<<<1, 1024, 0, s>>>(V);
    ctx.end_launch();
    TRY(ctx.launch_check("variant setup"));

    Original O{c_orig, obj_in, lo_orig, hi_orig, blo_orig, bhi_orig, col_scale, row_scale, base->objective_offset};
    Controls ctl{o->primal_tolerance, o->dual_tolerance, o->gap_tolerance, o->restart_reduction_factor,
                 o->primal_weight_smoothing, o->restart_every, o->restart_strategy, o->adaptive_step_size,
                 o->adaptive_primal_weight};
    TraceBuf tr{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const int poll_every = o->check_every_chunks > 0 ? o->check_every_chunks : 1;
    VarMixed M{};
    if (!mixed) {
        EngineVariants eng;
        eng.Bs = Bs;
        eng.V = V;
        eng.O = O;
        eng.grid = grid;
        TRY(run_chunks(ctx, eng, V.global, o->max_iterations, o->restart_every, poll_every, ctl, tr));
    } else {
        float* f_cv = static_cast<float*>(at(o_f_cv));
        float* f_rv = static_cast<float*>(at(o_f_rv));
        float* f_cn = static_cast<float*>(at(o_f_cn));
        float* f_rn = static_cast<float*>(at(o_f_rn));
        const int nbz = blocks_for(ctx, nnz + 16, kBlock) * 4;
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, cv, f_cv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<nbz, kBlock, 0, s>>>(nnz + 16, rv, f_rv);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<blocks_for(ctx, n, kBlock), kBlock, 0, s>>>(n, col_norm, f_cn);
        ctx.end_launch();
        ctx.begin_launch(MC_KERNEL_SETUP);
        k_to_float<<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(m, row_norm, f_rn);
        ctx.end_launch();
        M.cs = cs;
        M.ri = ri;
        M.cv = f_cv;
        M.rs = rs;
        M.ci = ci;
        M.rv = f_rv;
        M.col_norm = f_cn;
        M.row_norm = f_rn;
        M.c64 = c;
        M.blo64 = blo;
        M.bhi64 = bhi;
        M.xh = V.x;       // the FP64 start point is every variant's first base
        M.yh = V.y;
        M.axf = V.axb;
        M.atyf = V.xb;
        float* fn[7];
        for (int q = 0; q < 7; ++q) fn[q] = static_cast<float*>(at(o_fn[q]));
        float* fm[6];
        for (int q = 0; q < 6; ++q) fm[q] = static_cast<float*>(at(o_fm[q]));
        M.x = fn[0];
        M.xb = fn[1];
        M.xa = fn[2];
        M.g = fn[3];
        M.lo = fn[4];
        M.hi = fn[5];
        M.xdx = static_cast<float*>(at(o_fxdx));
        M.y = fm[0];
        M.ya = fm[1];
        M.axb = fm[2];
        M.yb = fm[3];
        M.rlo = fm[4];
        M.rhi = fm[5];
        // corrections start at zero (padding lanes included: gathers read them)
        for (int q = 0; q < 7; ++q) CU(cudaMemsetAsync(fn[q], 0, sizeof(float) * (size_t)nk, s));
        CU(cudaMemsetAsync(M.xdx, 0, sizeof(float) * 2 * (size_t)nk, s));
        for (int q = 0; q < 6; ++q) CU(cudaMemsetAsync(fm[q], 0, sizeof(float) * (size_t)mk, s));
        EngineVariantsMixed eng;
        eng.Bs = Bs;
        eng.V = V;
        eng.M = M;
        eng.O = O;
        eng.grid = grid;
        // the first correction LP of every running variant, around its start
        TRY(eng.residual_pass(ctx));
        TRY(eng.recenter(ctx, 1));
        TRY(run_chunks(ctx, eng, V.global, o->max_iterations, o->restart_every, poll_every, ctl, tr));
    }
    CU(cudaEventRecord(ctx.ev_c, s));

    // ---- outputs
    double* xo = static_cast<double*>(at(o_xo));
    double* yo = static_cast<double*>(at(o_yo));
    ctx.begin_launch(MC_KERNEL_OTHER);
    if (mixed) kvm_unscale_out<<<grid, kBlock, 0, s>>>(m, n, V, M, col_scale, row_scale, xo, yo);
    else kv_unscale_out<<<grid, kBlock, 0, s>>>(Bs, V, col_scale, row_scale, xo, yo);
    ctx.end_launch();
    TRY(ctx.launch_check("variant unscale"));
    for (int k = 0; k < count; ++k) {
        const int b = perm[k];
        if (x_out && x_out[b])
            CU(cudaMemcpyAsync(x_out[b], xo + (size_t)k * n, sizeof(double) * n, cudaMemcpyDefault, s));
        if (y_out && y_out[b])
            CU(cudaMemcpyAsync(y_out[b], yo + (size_t)k * m, sizeof(double) * m, cudaMemcpyDefault, s));
    }
    std::vector<DevState> hs(count + 2);
    CU(cudaMemcpyAsync(hs.data(), st, sizeof(DevState) * (count + 2), cudaMemcpyDeviceToHost, s));
    std::vector<int> hcert(2 * (size_t)count);
    CU(cudaMemcpyAsync(hcert.data(), V.cert_idx, sizeof(int) * hcert.size(), cudaMemcpyDeviceToHost, s));
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
    for (int k = 0; k < count; ++k) {
        const int b = perm[k];
        mc_pdlp_result& r = results[b];
        const DevState& S = hs[2 + k];
        r.status = S.status;
        r.objective = S.objective;
        r.primal_infeasibility = S.primal_infeas;
        r.dual_infeasibility = S.dual_infeas;
        r.duality_gap = S.gap;
        r.iterations = S.iter;
        r.certificate = S.status == MC_PDLP_INFEASIBLE_OR_UNBOUNDED ? S.cert : MC_CERT_NONE;
        r.certificate_index = r.certificate == MC_CERT_CROSSED_BOUNDS ? hcert[k]
                              : r.certificate == MC_CERT_ROW_ACTIVITY ? hcert[count + k]
                                                                      : -1;
        fill_message(&r, S.status == MC_PDLP_OPTIMAL ? "PDLP converged"
                         : r.certificate == MC_CERT_CROSSED_BOUNDS ? "infeasible: crossed variable bounds"
                         : r.certificate == MC_CERT_ROW_ACTIVITY ? "infeasible: row activity outside its bounds"
                         : r.certificate == MC_CERT_DUAL_RAY ? "infeasible: dual ray (Farkas certificate in dual)"
                         : S.status == MC_PDLP_NUMERICAL_FAILURE ? "non-finite iterate or residual"
                                                                 : "iteration limit reached");
        r.h2d_ms = dev_in ? 0.0 : h2d;
        r.kernel_ms = kern + (dev_in ? h2d : 0.0);
        r.d2h_ms = d2h;
        r.total_ms = total_ms;
        r.ruiz_iterations_executed = o->ruiz_scaling ? hs[0].ruiz_passes : 0;
        r.restarts = S.restarts;
        r.final_primal_weight = S.omega;
        r.final_step_size = S.eta;
        r.kernel_launches = total;
        r.refinement_rounds = mixed ? S.restarts : 0;  // each restart re-centres the variant's FP64 base
        r.inner_iterations = mixed ? S.iter : 0;
        for (int q = 0; q < MC_KERNEL_KINDS; ++q) {
            r.launches_by_kind[q] = ctx.launches[q];
            r.kernel_ms_by_kind[q] = ctx.kernel_ms[q];
        }
    }
    return MC_OK;
}

}  // namespace mc
