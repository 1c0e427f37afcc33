// Presolve and postsolve of a canonical model on the device
// (src/presolve/presolve.cpp:20-317).  Included once, by engine.cu after
// verify.cuh.
//
// The reference is a sequential scan: each pass removes the empty rows, then
// the empty columns, then walks the rows in order and, for a row left with a
// single entry, fixes that variable at once and substitutes it into the other
// rows -- so a singleton can make a later row of the same pass a singleton,
// and the right-hand sides change in the order of the walk.  The device
// version keeps those semantics exactly and does the work in parallel:
//
// * Empty rows / empty columns: one thread per line counts the entries that
//   survive the reference's filter (other end active, |a| > pivot
//   tolerance); a scan over the flags gives each removal its place on the
//   stack, in index order.  The first line that makes the model infeasible
//   or unbounded (atomicMin) cuts the step there, as the reference returns
//   there.
// * Row singletons run in rounds from a scan position P (all rows below P are
//   decided).  A round counts every row >= P; a row with one entry is a
//   tentative singleton, and among those with the same column only the first
//   fires (atomicMin per column; the later ones find the column fixed and
//   have no entry left).  A row r with c >= 2 entries of which h are fixed by
//   tentative singletons below it has c - h entries left at its turn; the
//   first such row with c - h = 1 is the boundary B (a singleton the round
//   did not foresee).  Every tentative singleton below B fires exactly as in
//   the sequential walk and no other row below B does (induction over the
//   rows: the singletons below a row are the tentative ones, so its count at
//   its turn is c - h), nothing at or above B is decided yet.  The round
//   commits the singletons below B, applies their substitutions, and moves P
//   to B.  Each round commits at least one singleton or ends the walk, so
//   rounds <= singletons + 1, and one round suffices when no singleton makes
//   another.  The rounds of a pass run inside one cooperative kernel
//   (kp_walk), with grid-wide barriers between their phases.
// * Substitutions: every row applies the fixes of the round that touch it in
//   the order of their singleton rows -- the order of the walk -- with the
//   same operands (rhs -= a * fixed, rounded separately), so the right-hand
//   sides are bit-identical.  The objective offset is summed in record order
//   on the host.
// * Postsolve: the LIFO pass of the reference computes each singleton's dual
//   from the duals of the other rows of its column as they are when the
//   record is popped: rows of the reduced model, rows removed later (already
//   restored) and rows removed earlier (still 0).  Records whose later-removed
//   rows are all restored run in parallel waves; the sums are double-double.
#pragma once

#include "engine.hpp"
#include "solve.cuh"
#include "verify.cuh"

#include <climits>
#include <cooperative_groups.h>
#include <map>
#include <mutex>
#include <vector>

namespace mc {

namespace cg = cooperative_groups;

constexpr int kNone = INT_MAX;

// Device control block of one presolve.
struct PsCtl {
    int stop;       // infeasible / unbounded found: every later kernel returns at once
    int status;     // mc_presolve_status
    int first_bad;  // step 1: first empty row with rhs != 0; step 3: first negative singleton
    int first_unb;  // step 2: first empty column with negative cost
    int boundary;   // step 3: first row a tentative singleton below it reduces
    int P;          // step 3 scan position
    int round;      // rounds so far (marks the columns fixed in a round)
    int cause;      // what stopped it: 0 empty row, 1 empty column, 2 negative singleton
    int nhit;       // rows listed in the walk's hit list this round
    int ntouch;     // rows listed in the walk's touched list this round
    long long rec;   // records on the stack
    long long inc;   // incident entries on the stack
    long long reductions;  // this pass
    long long stats[4];    // empty rows, empty cols, fixed vars, row singletons
};

struct PsRecords {
    int* kind;
    long long* index;
    long long* variable;
    double* value;
    double* value2;
    long long* inc_off;
    int* inc_len;
    long long* inc_row;
    double* inc_coef;
};

// --------------------------------------------------------------- step 1 / 2
// flag[i] = 1 for an active row with no surviving entry
__global__ void kp_empty_rows(int m, const int* __restrict__ rs, const int* __restrict__ ci,
                              const double* __restrict__ rv, const unsigned char* __restrict__ col_act,
                              const unsigned char* __restrict__ row_act, const double* __restrict__ rhs, double tol,
                              double feas, int* __restrict__ flag, PsCtl* __restrict__ ctl) {
    if (ctl->stop) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int f = 0;
        if (row_act[i]) {
            int cnt = 0;
            for (int p = rs[i]; p < rs[i + 1] && cnt == 0; ++p) cnt += col_act[ci[p]] && fabs(rv[p]) > tol;
            if (cnt == 0) {
                f = 1;
                if (fabs(rhs[i]) > feas) atomicMin(&ctl->first_bad, i);
            }
        }
        flag[i] = f;
    }
}

// pushes the empty rows below the first infeasible one (scan = inclusive scan of the flags)
__global__ void kp_push_rows(int m, const int* __restrict__ scan, const double* __restrict__ rhs,
                             unsigned char* __restrict__ row_act, PsRecords R, PsCtl* __restrict__ ctl) {
    if (ctl->stop) return;
    const int lim = min(ctl->first_bad, m);
    const long long base = ctl->rec;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
        const int before = i > 0 ? scan[i - 1] : 0;
        if (scan[i] == before) continue;
        const long long t = base + before;
        R.kind[t] = MC_RECORD_EMPTY_ROW;
        R.index[t] = i;
        R.variable[t] = -1;
        R.value[t] = rhs[i];
        R.value2[t] = 0.0;
        R.inc_len[t] = 0;
        row_act[i] = 0;
    }
}

__global__ void kp_empty_cols(int n, const int* __restrict__ cs, const int* __restrict__ ri,
                              const double* __restrict__ v, const unsigned char* __restrict__ row_act,
                              const unsigned char* __restrict__ col_act, const double* __restrict__ obj, double tol,
                              double dual_tol, int* __restrict__ flag, PsCtl* __restrict__ ctl) {
    if (ctl->stop) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        int f = 0;
        if (col_act[j]) {
            int cnt = 0;
            for (int p = cs[j]; p < cs[j + 1] && cnt == 0; ++p) cnt += row_act[ri[p]] && fabs(v[p]) > tol;
            if (cnt == 0) {
                f = 1;
                if (obj[j] < -dual_tol) atomicMin(&ctl->first_unb, j);
            }
        }
        flag[j] = f;
    }
}

__global__ void kp_push_cols(int n, const int* __restrict__ scan, const double* __restrict__ obj,
                             unsigned char* __restrict__ col_act, PsRecords R, PsCtl* __restrict__ ctl) {
    if (ctl->stop) return;
    const int lim = min(ctl->first_unb, n);
    const long long base = ctl->rec;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lim; j += gridDim.x * blockDim.x) {
        const int before = j > 0 ? scan[j - 1] : 0;
        if (scan[j] == before) continue;
        const long long t = base + before;
        R.kind[t] = MC_RECORD_EMPTY_COLUMN;
        R.index[t] = j;
        R.variable[t] = -1;
        R.value[t] = obj[j];
        R.value2[t] = 0.0;
        R.inc_len[t] = 0;
        col_act[j] = 0;
    }
}

// closes step 1 (which = 0) or step 2 (which = 1): counts, statistics, stop
__global__ void kp_close_step(int which, int len, const int* __restrict__ scan, PsCtl* __restrict__ ctl) {
    if (ctl->stop) return;
    const int bad = which == 0 ? ctl->first_bad : ctl->first_unb;
    const int lim = min(bad, len);
    const long long cnt = lim > 0 ? scan[lim - 1] : 0;
    ctl->rec += cnt;
    ctl->reductions += cnt;
    ctl->stats[which] += cnt;
    if (bad != kNone) {
        ctl->stop = 1;
        ctl->cause = which;
        ctl->status = which == 0 ? MC_PRESOLVE_INFEASIBLE : MC_PRESOLVE_UNBOUNDED;
    }
}

// ------------------------------------------------------------------ step 3
// The singleton walk of one pass is one cooperative kernel: each block owns a
// contiguous range of rows, the phases of a round are separated by grid-wide
// barriers, and the rounds repeat on the device until the walk ends (at most
// m + 1 rounds; each round commits a singleton or ends the walk).  Phases:
//   1 counts of the rows >= P (every row in a pass's first round, later the
//     counts the substitutions keep) and bids of one-entry rows for their
//     column (atomicMin: the first bidder is the tentative singleton); each
//     block lists its bidders in row order;
//   2 tentative singletons (over the bidder lists); hits on the later rows of
//     their columns (a row hit for the first time joins the hit list); the
//     first singleton whose value would be negative;
//   3 the boundary (over the hit list: the first row the hits leave with one
//     entry); bids cleared;
//   4 the limit L = min(boundary, first negative, m); singletons per block;
//     hits cleared;
//   5 commit below L in row order (block prefix + block scan over the
//     bidder list), incident counts;
//   6 incident lists in stack order; touched rows listed;
//   7 substitutions in the touched rows, counts kept; the round closed.
struct Walk {
    int m;
    const int *rs, *ci;
    const double* rv;
    const int *cs, *ri;
    const double* v;
    const double* obj;
    unsigned char *row_act, *col_act, *fire;
    int *cnt, *hits, *sc, *col_first, *fix_round, *fix_row, *fire_col, *inc_cnt, *touched;
    double *sa, *fix_val, *rhs;
    int *block_fires, *block_inc;
    int *bid_list, *hit_list, *touch_list;  // [m] each
    double tol, feas;
    PsRecords R;
    PsCtl* ctl;
};

constexpr int kWalkThreads = 256;
constexpr int kWalkWarps = kWalkThreads / 32;

// Exclusive prefix of v over the block's threads in thread order; *total
// receives the block's sum.  Every thread of the block must call it.
__device__ __forceinline__ int block_exclusive(int v, int* sh, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kWalkWarps ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWalkWarps) sh[lane] = w;
    }
    __syncthreads();
    const int before = (warp > 0 ? sh[warp - 1] : 0) + x - v;
    *total = sh[kWalkWarps - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kWalkThreads) kp_walk(Walk W) {
    __shared__ int sh[32];
    cg::grid_group grid = cg::this_grid();
    PsCtl* ctl = W.ctl;
    if (ctl->stop) return;  // set before the launch: the same for every block
    const int m = W.m, nb = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const int gtid = b * kWalkThreads + tid, gthreads = nb * kWalkThreads;
    const int per = (m + nb - 1) / nb;
    const int lo = min(b * per, m), hi = min(lo + per, m);
    const double tol = W.tol;
    int* bids = W.bid_list + lo;  // this block's bidders, ascending (at most hi - lo)
    for (int it = 0; it <= m; ++it) {
        const int P = ctl->P, round = ctl->round;
        const int r0 = max(lo, P);
        // the lists of the last round are read by every block before the
        // barrier that ended it, so they restart here (appends come after
        // the next barrier)
        if (b == 0 && tid == 0) {
            ctl->nhit = 0;
            ctl->ntouch = 0;
        }
        // 1. counts (every row in the pass's first round, later the kept
        //    counts) and bids; the block's bidders listed in row order
        int nbid = 0;
        for (int base = r0; base < hi; base += kWalkThreads) {
            const int i = base + tid;
            int f = 0;
            if (i < hi) {
                if (it == 0) {
                    W.hits[i] = 0;
                    int c = 0, j = -1;
                    double a = 0.0;
                    if (W.row_act[i])
                        for (int p = W.rs[i]; p < W.rs[i + 1]; ++p)
                            if (W.col_act[W.ci[p]] && fabs(W.rv[p]) > tol) {
                                ++c;
                                j = W.ci[p];
                                a = W.rv[p];
                            }
                    W.cnt[i] = c;
                    if (c == 1) {
                        W.sc[i] = j;
                        W.sa[i] = a;
                    }
                }
                f = W.row_act[i] && W.cnt[i] == 1;
            }
            int t = 0;
            const int ex = block_exclusive(f, sh, &t);
            if (f) {
                bids[nbid + ex] = i;
                atomicMin(&W.col_first[W.sc[i]], i);
            }
            nbid += t;
        }
        grid.sync();
        // 2. tentative singletons, hits on the later rows of their columns
        //    (rows hit for the first time listed), first negative value
        for (int k = tid; k < nbid; k += kWalkThreads) {
            const int i = bids[k];
            const bool f = W.col_first[W.sc[i]] == i;
            W.fire[i] = f;
            if (!f) continue;
            if (__ddiv_rn(W.rhs[i], W.sa[i]) < -W.feas) atomicMin(&ctl->first_bad, i);
            const int j = W.sc[i];
            for (int p = W.cs[j]; p < W.cs[j + 1]; ++p) {
                const int r = W.ri[p];
                if (r > i && W.row_act[r] && W.cnt[r] >= 2 && fabs(W.v[p]) > tol)
                    if (atomicAdd(&W.hits[r], 1) == 0) W.hit_list[atomicAdd(&ctl->nhit, 1)] = r;
            }
        }
        grid.sync();
        // 3. boundary (the first row the hits leave with one entry); bids cleared
        for (int k = tid; k < nbid; k += kWalkThreads) W.col_first[W.sc[bids[k]]] = kNone;
        const int nhit = ctl->nhit;
        for (int k = gtid; k < nhit; k += gthreads) {
            const int r = W.hit_list[k];
            if (W.cnt[r] - W.hits[r] == 1) atomicMin(&ctl->boundary, r);
        }
        grid.sync();
        // 4. the limit; singletons of this block below it; hits cleared
        const int fb = ctl->first_bad;
        const int L = min(min(ctl->boundary, fb), m);
        const long long rec0 = ctl->rec, inc0 = ctl->inc;
        for (int k = gtid; k < nhit; k += gthreads) W.hits[W.hit_list[k]] = 0;
        int mine = 0, tot = 0;
        for (int k = tid; k < nbid; k += kWalkThreads) {
            const int i = bids[k];
            mine += (i < L && W.fire[i]) ? 1 : 0;
        }
        block_exclusive(mine, sh, &tot);
        if (tid == 0) W.block_fires[b] = tot;
        grid.sync();
        // 5. commit in row order: ranks from the earlier blocks' counts and a
        //    block scan over the (ascending) bidder list
        int pre = 0, all = 0;
        for (int q = tid; q < nb; q += kWalkThreads) {
            const int c = W.block_fires[q];
            if (q < b) pre += c;
            all += c;
        }
        block_exclusive(pre, sh, &pre);
        int nf = 0;
        block_exclusive(all, sh, &nf);
        const int myfires = W.block_fires[b];
        int run = 0, my_inc = 0;
        for (int base = 0; base < nbid; base += kWalkThreads) {
            const int k = base + tid;
            const int i = k < nbid ? bids[k] : 0;
            const int f = (k < nbid && i < L && W.fire[i]) ? 1 : 0;
            int t = 0;
            const int ex = block_exclusive(f, sh, &t);
            if (f) {
                const int q = pre + run + ex;
                const int j = W.sc[i];
                double fixed = __ddiv_rn(W.rhs[i], W.sa[i]);
                if (fixed < 0.0) fixed = 0.0;
                const long long rt = rec0 + 2LL * q;
                W.R.kind[rt] = MC_RECORD_ROW_SINGLETON;
                W.R.index[rt] = i;
                W.R.variable[rt] = j;
                W.R.value[rt] = W.sa[i];
                W.R.value2[rt] = W.rhs[i];
                W.R.inc_len[rt] = 0;
                W.R.kind[rt + 1] = MC_RECORD_FIXED_VARIABLE;
                W.R.index[rt + 1] = j;
                W.R.variable[rt + 1] = -1;
                W.R.value[rt + 1] = fixed;
                W.R.value2[rt + 1] = W.obj[j];
                W.row_act[i] = 0;
                W.col_act[j] = 0;
                W.fix_round[j] = round;
                W.fix_row[j] = i;
                W.fix_val[j] = fixed;
                W.fire_col[q] = j;
                // the rows this fix reaches: no other singleton of the round
                // has an entry in column j, so their activity is settled here
                int c = 0;
                for (int p = W.cs[j]; p < W.cs[j + 1]; ++p) {
                    const int r = W.ri[p];
                    c += r != i && W.row_act[r] && fabs(W.v[p]) > tol;
                }
                W.inc_cnt[q] = c;
                my_inc += c;
            }
            run += t;
        }
        int inc_tot = 0;
        block_exclusive(my_inc, sh, &inc_tot);
        if (tid == 0) W.block_inc[b] = inc_tot;
        grid.sync();
        // 6. incident lists (column order), in stack order; touched rows listed
        int ipre = 0, iall = 0;
        for (int q = tid; q < nb; q += kWalkThreads) {
            const int c = W.block_inc[q];
            if (q < b) ipre += c;
            iall += c;
        }
        block_exclusive(ipre, sh, &ipre);
        int inc_all = 0;
        block_exclusive(iall, sh, &inc_all);
        run = 0;
        for (int base = 0; base < myfires; base += kWalkThreads) {
            const int k = base + tid;
            const int q = pre + k;
            const int c = k < myfires ? W.inc_cnt[q] : 0;
            int t = 0;
            const int ex = block_exclusive(c, sh, &t);
            if (k < myfires) {
                const long long off = inc0 + ipre + run + ex;
                const int j = W.fire_col[q];
                long long w = off;
                for (int p = W.cs[j]; p < W.cs[j + 1] && w < off + c; ++p) {
                    const int r = W.ri[p];
                    if (W.row_act[r] && fabs(W.v[p]) > tol) {
                        W.R.inc_row[w] = r;
                        W.R.inc_coef[w] = W.v[p];
                        if (atomicExch(&W.touched[r], round) != round) W.touch_list[atomicAdd(&ctl->ntouch, 1)] = r;
                        ++w;
                    }
                }
                const long long rt = rec0 + 2LL * q + 1;
                W.R.inc_off[rt] = off;
                W.R.inc_len[rt] = (int)(w - off);
            }
            run += t;
        }
        grid.sync();
        // 7. substitutions in the order of the singleton rows
        //    (presolve.cpp:155-159), a warp per touched row: each pass takes
        //    the round's fix of the smallest singleton row above the last one
        const int ntouch = ctl->ntouch;
        {
            const int lane = tid & 31;
            for (int k = gtid >> 5; k < ntouch; k += gthreads >> 5) {
                const int r = W.touch_list[k];
                const int bb = W.rs[r], e = W.rs[r + 1];
                int kf = 0;
                for (int p = bb + lane; p < e; p += 32) kf += W.fix_round[W.ci[p]] == round && fabs(W.rv[p]) > tol;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) kf += __shfl_xor_sync(0xffffffffu, kf, o);
                if (kf == 0) continue;
                const int left = W.cnt[r] - kf;
                if (left == 1)
                    for (int p = bb + lane; p < e; p += 32)
                        if (W.col_act[W.ci[p]] && fabs(W.rv[p]) > tol) {
                            W.sc[r] = W.ci[p];
                            W.sa[r] = W.rv[p];
                        }
                double h = W.rhs[r];
                int last = -1;
                for (int t = 0; t < kf; ++t) {
                    int best = kNone;
                    double a = 0.0, f = 0.0;
                    for (int p = bb + lane; p < e; p += 32) {
                        const int c = W.ci[p];
                        if (W.fix_round[c] != round || !(fabs(W.rv[p]) > tol)) continue;
                        const int fr = W.fix_row[c];
                        if (fr > last && fr < best) {
                            best = fr;
                            a = W.rv[p];
                            f = W.fix_val[c];
                        }
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        const int ob = __shfl_xor_sync(0xffffffffu, best, o);
                        const double oa = __shfl_xor_sync(0xffffffffu, a, o);
                        const double of = __shfl_xor_sync(0xffffffffu, f, o);
                        if (ob < best) {
                            best = ob;
                            a = oa;
                            f = of;
                        }
                    }
                    h = __dsub_rn(h, __dmul_rn(a, f));
                    last = best;
                }
                if (lane == 0) {
                    W.cnt[r] = left;
                    W.rhs[r] = h;
                }
            }
        }
        if (b == 0 && tid == 0) {  // close the round (the other blocks read no control field it writes until the barrier)
            ctl->rec = rec0 + 2LL * nf;
            ctl->inc = inc0 + inc_all;
            ctl->reductions += nf;
            ctl->stats[2] += nf;
            ctl->stats[3] += nf;
            ctl->round = round + 1;
            if (fb != kNone && fb == L) {  // presolve.cpp:137-142
                ctl->stop = 1;
                ctl->cause = 2;
                ctl->status = MC_PRESOLVE_INFEASIBLE;
            } else {
                ctl->P = L;
                ctl->boundary = kNone;
                ctl->first_bad = kNone;
            }
        }
        grid.sync();
        if (ctl->stop || ctl->P >= m) break;
    }
}

__global__ void kp_begin_pass(PsCtl* __restrict__ ctl) {
    ctl->reductions = 0;
    ctl->first_bad = ctl->first_unb = ctl->boundary = kNone;
    ctl->P = 0;
}

__global__ void kp_check_finite(const double* __restrict__ a, long long len, int* __restrict__ bad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
         i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(a[i])) atomicOr(bad, 1);
}

// ------------------------------------------------------------- compaction
__global__ void kp_flag_active(int len, const unsigned char* __restrict__ act, int* __restrict__ flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) flag[i] = act[i];
}

__global__ void kp_compact_rows(int m, const unsigned char* __restrict__ row_act, const int* __restrict__ scan,
                                const double* __restrict__ rhs, int* __restrict__ new_row,
                                long long* __restrict__ row_map, double* __restrict__ rhs_out,
                                int* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (!row_act[i]) {
            new_row[i] = -1;
            continue;
        }
        const int q = scan[i] - 1;
        new_row[i] = q;
        row_map[q] = i;
        rhs_out[q] = rhs[i];
        if (!isfinite(rhs[i])) atomicOr(bad, 1);
    }
}

// surviving entries of each active column (0 for removed columns)
__global__ void kp_col_counts(int n, const int* __restrict__ cs, const int* __restrict__ ri,
                              const double* __restrict__ v, const unsigned char* __restrict__ row_act,
                              const unsigned char* __restrict__ col_act, double tol, int* __restrict__ cc) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        int c = 0;
        if (col_act[j])
            for (int p = cs[j]; p < cs[j + 1]; ++p) c += row_act[ri[p]] && fabs(v[p]) > tol;
        cc[j] = c;
    }
}

__global__ void kp_compact_cols(int n, const int* __restrict__ cs, const int* __restrict__ ri,
                                const double* __restrict__ v, const unsigned char* __restrict__ row_act,
                                const unsigned char* __restrict__ col_act, double tol,
                                const int* __restrict__ col_scan, const int* __restrict__ cc_scan,
                                const int* __restrict__ new_row, const double* __restrict__ obj,
                                int* __restrict__ cs_out, int* __restrict__ ri_out, double* __restrict__ v_out,
                                double* __restrict__ obj_out, long long* __restrict__ col_map) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (!col_act[j]) continue;
        const int q = col_scan[j] - 1;
        col_map[q] = j;
        obj_out[q] = obj[j];
        cs_out[q + 1] = cc_scan[j];
        int w = j > 0 ? cc_scan[j - 1] : 0;
        for (int p = cs[j]; p < cs[j + 1]; ++p)
            if (row_act[ri[p]] && fabs(v[p]) > tol) {
                ri_out[w] = new_row[ri[p]];
                v_out[w] = v[p];
                ++w;
            }
    }
}

// ---------------------------------------------------------------- postsolve
__global__ void kp_post_zero(int m, int n, double* __restrict__ x, double* __restrict__ y) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (long long j = t0; j < n; j += stride) x[j] = 0.0;
    for (long long i = t0; i < m; i += stride) y[i] = 0.0;
}

__global__ void kp_post_place(long long pm, long long pn, const long long* __restrict__ row_map,
                              const long long* __restrict__ col_map, const double* __restrict__ rx, long long rx_len,
                              const double* __restrict__ ry, long long ry_len, double* __restrict__ x,
                              double* __restrict__ y) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (long long q = t0; q < pn && q < rx_len; q += stride) x[col_map[q]] = rx[q];
    for (long long q = t0; q < pm && q < ry_len; q += stride) y[row_map[q]] = ry[q];
}

// primal values of removed columns; the stack position of every singleton row
__global__ void kp_post_records(long long nrec, PsRecords R, double* __restrict__ x, int* __restrict__ pos) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrec;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = R.kind[t];
        if (k == MC_RECORD_EMPTY_COLUMN) x[R.index[t]] = R.value2[t];
        else if (k == MC_RECORD_FIXED_VARIABLE) x[R.index[t]] = R.value[t];
        else if (k == MC_RECORD_ROW_SINGLETON) pos[R.index[t]] = (int)t;
    }
}

// One wave of singleton duals: a record is ready when every row of its
// column removed after it (popped before it) is restored; it reads those
// restored duals, the reduced model's duals, and 0 for rows removed before
// it.  pi = (c_k - sum_{r != i} a_rk y_r) / a_ik (presolve.cpp:280-298).
__global__ void kp_post_wave(int nsing, const int* __restrict__ sing, PsRecords R, const int* __restrict__ cs,
                             const int* __restrict__ ri, const double* __restrict__ v, const double* __restrict__ obj,
                             const int* __restrict__ pos, const unsigned char* __restrict__ done,
                             const double* __restrict__ y, const double* __restrict__ pi_in,
                             double* __restrict__ pi_out, unsigned char* __restrict__ now_done,
                             int* __restrict__ counters) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nsing; q += gridDim.x * blockDim.x) {
        const int t = sing[q];
        const int i = (int)R.index[t];
        if (done[i]) continue;
        const int k = (int)R.variable[t];
        bool ready = true;
        for (int p = cs[k]; p < cs[k + 1] && ready; ++p) {
            const int r = ri[p];
            if (r != i && pos[r] > t && !done[r]) ready = false;
        }
        if (!ready) {
            atomicAdd(&counters[0], 1);
            continue;
        }
        DD s{0.0, 0.0};
        for (int p = cs[k]; p < cs[k + 1]; ++p) {
            const int r = ri[p];
            if (r == i) continue;
            const double d = pos[r] < 0 ? y[r] : (pos[r] > t ? pi_in[r] : 0.0);
            s = dd_add_product(s, v[p], d);
        }
        // (c_k - s) / a in double-double, rounded once
        const DD num = dd_add(DD{obj[k], 0.0}, DD{-s.hi, -s.lo});
        const double a = R.value[t];
        const double q1 = num.hi / a;
        const double rem = __fma_rn(-q1, a, num.hi) + num.lo;
        const double pi = q1 + rem / a;
        if (!isfinite(pi)) atomicOr(&counters[1], 1);
        pi_out[i] = pi;
        now_done[i] = 1;
    }
}

__global__ void kp_post_mark(int nsing, const int* __restrict__ sing, PsRecords R,
                             unsigned char* __restrict__ now_done, unsigned char* __restrict__ done,
                             const double* __restrict__ pi_out, double* __restrict__ pi_in) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nsing; q += gridDim.x * blockDim.x) {
        const int i = (int)R.index[sing[q]];
        if (now_done[i]) {
            now_done[i] = 0;
            done[i] = 1;
            pi_in[i] = pi_out[i];
        }
    }
}

__global__ void kp_post_duals(int nsing, const int* __restrict__ sing, PsRecords R, const double* __restrict__ pi,
                              double* __restrict__ y) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nsing; q += gridDim.x * blockDim.x) {
        const int i = (int)R.index[sing[q]];
        y[i] = pi[i];
    }
}

// block partials of sum c_j x_j in double-double, in a fixed order
__global__ void kp_post_objective(int n, const double* __restrict__ obj, const double* __restrict__ x,
                                  DD* __restrict__ parts) {
    __shared__ DD sh[kBlock];
    DD s{0.0, 0.0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        s = dd_add_product(s, obj[j], x[j]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = dd_add(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) parts[blockIdx.x] = sh[0];
}

}  // namespace mc

// ------------------------------------------------------------ host driver
struct mc_presolve {
    int device = -1;
    mc_presolve_info info{};
    // the input model (kept for postsolve)
    int m = 0, n = 0;
    long long nnz = 0;
    int *cs = nullptr, *ri = nullptr;
    double *v = nullptr, *obj = nullptr;
    double offset = 0.0;
    // the reduced model and maps
    int *cs_out = nullptr, *ri_out = nullptr;
    double *v_out = nullptr, *rhs_out = nullptr, *obj_out = nullptr;
    long long *row_map = nullptr, *col_map = nullptr;
    // the stack
    mc::PsRecords R{};
    std::vector<void*> owned;
};

namespace mc {

// A stream-ordered memory pool per device for presolve results and scratch.
// Freed blocks stay reserved (up to 1 GiB) for the next call instead of
// being unmapped at every synchronisation: repeated presolves then allocate
// in microseconds.  Pools live until the process exits; where one cannot be
// made, the device's default pool is used.
inline cudaMemPool_t ps_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> guard(mu);
    const auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        pool = nullptr;
    } else {
        unsigned long long keep = 1ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pools[device] = pool;
    return pool;
}

inline cudaError_t ps_malloc(void** ptr, size_t bytes, int device, cudaStream_t s) {
    const cudaMemPool_t pool = ps_pool(device);
    return pool ? cudaMallocFromPoolAsync(ptr, bytes, pool, s) : cudaMallocAsync(ptr, bytes, s);
}

inline int ps_alloc(mc_presolve* p, void** ptr, size_t bytes, cudaStream_t s) {
    if (ps_malloc(ptr, bytes < 16 ? 16 : bytes, p->device, s) != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        return set_error(MC_ERR_OUT_OF_MEMORY, "presolve buffer (%zu bytes)", bytes);
    }
    p->owned.push_back(*ptr);
    return MC_OK;
}

// Frees a result: its buffers go back to the pool (ordered on the device's
// default stream; every call that wrote them has synchronised).
inline void ps_free(mc_presolve* p) {
    if (!p) return;
    if (p->device >= 0) cudaSetDevice(p->device);
    for (void* q : p->owned) cudaFreeAsync(q, 0);
    delete p;
}

}  // namespace mc

namespace mc {

// Scratch on the context's stream, released when the call ends.
struct PsScratch {
    cudaStream_t s;
    int device;
    std::vector<void*> ptrs;
    int rc = MC_OK;
    PsScratch(cudaStream_t st, int dev) : s(st), device(dev) {}
    template <class T>
    void get(T** ptr, size_t count) {
        *ptr = nullptr;
        if (rc != MC_OK) return;
        if (ps_malloc(reinterpret_cast<void**>(ptr), (count < 2 ? 2 : count) * sizeof(T), device, s) != cudaSuccess) {
            *ptr = nullptr;
            cudaGetLastError();
            rc = set_error(MC_ERR_OUT_OF_MEMORY, "presolve scratch (%zu bytes)", count * sizeof(T));
            return;
        }
        ptrs.push_back(*ptr);
    }
    ~PsScratch() {
        for (void* q : ptrs) cudaFreeAsync(q, s);
        cudaStreamSynchronize(s);
    }
};

int presolve_body(Ctx& ctx, const mc_canonical_lp* lp, const mc_presolve_options* o, mc_presolve* P) {
    cudaStream_t s = ctx.stream;
    const int m = lp->num_rows, n = lp->num_cols;
    const long long nnz = lp->nnz;
    const size_t mm = (size_t)m + 1, nn = (size_t)n + 1, zz = (size_t)nnz + 1;
    {
        int rc = MC_OK;
        auto own = [&](auto** ptr, size_t count) {
            if (rc == MC_OK) rc = ps_alloc(P, reinterpret_cast<void**>(ptr), count * sizeof(**ptr), s);
        };
        own(&P->cs, nn);
        own(&P->ri, zz);
        own(&P->v, zz);
        own(&P->obj, nn);
        own(&P->cs_out, nn);
        own(&P->ri_out, zz);
        own(&P->v_out, zz);
        own(&P->rhs_out, mm);
        own(&P->obj_out, nn);
        own(&P->row_map, mm);
        own(&P->col_map, nn);
        const size_t rr = mm + nn;  // every line leaves at most one record
        own(&P->R.kind, rr);
        own(&P->R.index, rr);
        own(&P->R.variable, rr);
        own(&P->R.value, rr);
        own(&P->R.value2, rr);
        own(&P->R.inc_off, rr);
        own(&P->R.inc_len, rr);
        own(&P->R.inc_row, zz);
        own(&P->R.inc_coef, zz);
        TRY(rc);
    }
    PsScratch S(s, ctx.device);
    const size_t lines = (size_t)std::max(m, n) + 1;
    int *rs, *ci, *cursor, *long_rows, *counters, *scan_tmp, *cnt, *hits, *sc, *col_first, *flag, *fix_round,
        *fix_row, *fire_col, *inc_cnt, *new_row, *cc, *touched;
    double *rv, *rhs, *sa, *fix_val;
    unsigned char *row_act, *col_act, *fire;
    PsCtl* ctl;
    S.get(&rs, mm);
    S.get(&ci, zz);
    S.get(&rv, zz);
    S.get(&cursor, mm);
    S.get(&long_rows, mm);
    S.get(&counters, 4);
    S.get(&scan_tmp, lines / kScanTile + 4096);
    S.get(&rhs, mm);
    S.get(&sa, mm);
    S.get(&fix_val, nn);
    S.get(&row_act, mm);
    S.get(&col_act, nn);
    S.get(&fire, mm);
    S.get(&cnt, mm);
    S.get(&hits, mm);
    S.get(&touched, mm);
    S.get(&sc, mm);
    S.get(&col_first, nn);
    S.get(&flag, lines);
    S.get(&fix_round, nn);
    S.get(&fix_row, nn);
    S.get(&fire_col, mm);
    S.get(&inc_cnt, mm);
    S.get(&new_row, mm);
    S.get(&cc, nn);
    S.get(&ctl, 1);
    TRY(S.rc);

    // the input, checked as SparseCanonicalModel::validate does
    // (src/transform/sparse_canonicalize.cpp:20-37), without the size cap
    const cudaMemcpyKind kind = cudaMemcpyDefault;
    if (cudaMemcpyAsync(P->cs, lp->col_start, sizeof(int) * nn, kind, s) != cudaSuccess ||
        (nnz > 0 && (cudaMemcpyAsync(P->ri, lp->row_index, sizeof(int) * nnz, kind, s) != cudaSuccess ||
                     cudaMemcpyAsync(P->v, lp->value, sizeof(double) * nnz, kind, s) != cudaSuccess)) ||
        (n > 0 && cudaMemcpyAsync(P->obj, lp->objective, sizeof(double) * n, kind, s) != cudaSuccess) ||
        (m > 0 && cudaMemcpyAsync(rhs, lp->rhs, sizeof(double) * m, kind, s) != cudaSuccess)) {
        cudaGetLastError();
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve: cannot read the model arrays");
    }
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    if (n > 0)
        k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, nnz, P->cs, P->ri, P->v, counters + 2);
    if (m > 0) kp_check_finite<<<blocks_for(ctx, m, kBlock), kBlock, 0, s>>>(rhs, m, counters + 3);
    if (n > 0) kp_check_finite<<<blocks_for(ctx, n, kBlock), kBlock, 0, s>>>(P->obj, n, counters + 3);
    {
        int hc[2] = {0, 0}, h0 = 0;
        CU(cudaMemcpyAsync(hc, counters + 2, sizeof hc, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(&h0, P->cs, sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        TRY(ctx.launch_check("presolve validation"));
        if (hc[0] || (n == 0 && (h0 != 0 || nnz != 0)))
            return set_error(MC_ERR_INVALID_ARGUMENT, "invalid canonical CSC (flags %d)", hc[0]);
        if (hc[1]) return set_error(MC_ERR_INVALID_ARGUMENT, "canonical rhs or objective non-finite");
    }
    mc_presolve_info& I = P->info;
    I.status = MC_PRESOLVE_OPTIMAL;
    I.original_rows = m;
    I.original_cols = n;
    // rows in ascending column order, as the reference lists them (presolve.cpp:49-58)
    if (m > 0 && n > 0) {
        TRY(build_csr(ctx, m, n, nnz, P->cs, P->ri, P->v, rs, ci, rv, cursor, long_rows, counters, scan_tmp));
    } else if (m > 0) {
        CU(cudaMemsetAsync(rs, 0, sizeof(int) * mm, s));
    }
    CU(cudaMemsetAsync(row_act, 1, mm, s));
    CU(cudaMemsetAsync(col_act, 1, nn, s));
    CU(cudaMemsetAsync(col_first, 0x7f, sizeof(int) * nn, s));  // above every row index
    CU(cudaMemsetAsync(fix_round, 0xff, sizeof(int) * nn, s));  // -1
    CU(cudaMemsetAsync(touched, 0xff, sizeof(int) * mm, s));
    CU(cudaMemsetAsync(cnt, 0, sizeof(int) * mm, s));
    CU(cudaMemsetAsync(ctl, 0, sizeof(PsCtl), s));
    const double tol = o->pivot_tolerance;
    const int gm = blocks_for(ctx, std::max(m, 1), kBlock), gn = blocks_for(ctx, std::max(n, 1), kBlock);
    const PsRecords R = P->R;
    // the singleton walk: one cooperative kernel per pass, its grid at most
    // the co-resident blocks (four per SM at most), and no more than one per
    // 512 rows: a small model's barriers then span few blocks
    int walk_per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&walk_per_sm, kp_walk, kWalkThreads, 0));
    const int walk_blocks = std::max(1, std::min(std::max(1, std::min(walk_per_sm, 4)) * ctx.sm_count, (m + 511) / 512));
    int *block_fires = nullptr, *block_inc = nullptr, *bid_list = nullptr, *hit_list = nullptr,
        *touch_list = nullptr;
    S.get(&block_fires, (size_t)walk_blocks);
    S.get(&block_inc, (size_t)walk_blocks);
    S.get(&bid_list, mm);
    S.get(&hit_list, mm);
    S.get(&touch_list, mm);
    TRY(S.rc);
    Walk W{m, rs, ci, rv, P->cs, P->ri, P->v, P->obj, row_act, col_act, fire, cnt, hits, sc, col_first, fix_round,
           fix_row, fire_col, inc_cnt, touched, sa, fix_val, rhs, block_fires, block_inc, bid_list, hit_list,
           touch_list, tol, o->feasibility_tolerance, R, ctl};
    PsCtl h{};
    long long pass = 0, rounds = 0;
    for (; pass < o->max_passes; ++pass) {
        ctx.begin_launch(MC_KERNEL_OTHER);
        kp_begin_pass<<<1, 1, 0, s>>>(ctl);
        ctx.end_launch();
        if (m > 0) {  // 1. empty rows (presolve.cpp:64-88)
            kp_empty_rows<<<gm, kBlock, 0, s>>>(m, rs, ci, rv, col_act, row_act, rhs, tol, o->feasibility_tolerance,
                                                flag, ctl);
            inclusive_scan(ctx, flag, m, scan_tmp, MC_KERNEL_OTHER);
            kp_push_rows<<<gm, kBlock, 0, s>>>(m, flag, rhs, row_act, R, ctl);
            kp_close_step<<<1, 1, 0, s>>>(0, m, flag, ctl);
        }
        if (n > 0) {  // 2. empty columns (presolve.cpp:90-114)
            kp_empty_cols<<<gn, kBlock, 0, s>>>(n, P->cs, P->ri, P->v, row_act, col_act, P->obj, tol,
                                                o->dual_tolerance, flag, ctl);
            inclusive_scan(ctx, flag, n, scan_tmp, MC_KERNEL_OTHER);
            kp_push_cols<<<gn, kBlock, 0, s>>>(n, flag, P->obj, col_act, R, ctl);
            kp_close_step<<<1, 1, 0, s>>>(1, n, flag, ctl);
        }
        // 3. row singletons (presolve.cpp:119-167), in rounds on the device
        if (m > 0) {
            void* args[] = {&W};
            ctx.begin_launch(MC_KERNEL_OTHER);
            CU(cudaLaunchCooperativeKernel((const void*)kp_walk, dim3(walk_blocks), dim3(kWalkThreads), args, 0, s));
            ctx.end_launch();
        }
        CU(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        TRY(ctx.launch_check("presolve pass"));
        if (m > 0 && !h.stop && h.P < m) return set_error(MC_ERR_INTERNAL, "presolve: singleton walk did not end");
        rounds = h.round;
        if (h.stop || h.reductions == 0) break;
    }
    I.empty_rows_removed = h.stats[0];
    I.empty_cols_removed = h.stats[1];
    I.fixed_vars_removed = h.stats[2];
    I.row_singletons_removed = h.stats[3];
    I.records = h.rec;
    I.incident_entries = h.inc;
    I.scan_rounds = rounds;
    CU(cudaMemsetAsync(P->cs_out, 0, sizeof(int), s));
    if (h.stop) {
        // the reference returns there: statistics' pass count 0, default
        // (empty) model (presolve.cpp:80-84, 106-110, 137-142)
        static const char* const why[3] = {
            "presolve: empty row with non-zero RHS detected", "presolve: empty column with negative cost detected",
            "presolve: row singleton implies negative value for canonical non-negative variable"};
        I.status = h.status;
        std::snprintf(I.message, sizeof I.message, "%s", why[h.cause < 0 || h.cause > 2 ? 0 : h.cause]);
        I.passes_executed = 0;
        I.objective_offset = 0.0;
        return MC_OK;
    }
    I.passes_executed = pass;
    // compaction (presolve.cpp:172-209)
    int nm = 0, nc = 0, nz = 0, hb = 0;
    CU(cudaMemsetAsync(counters, 0, sizeof(int) * 4, s));
    if (m > 0) {
        kp_flag_active<<<gm, kBlock, 0, s>>>(m, row_act, flag);
        inclusive_scan(ctx, flag, m, scan_tmp, MC_KERNEL_OTHER);
        kp_compact_rows<<<gm, kBlock, 0, s>>>(m, row_act, flag, rhs, new_row, P->row_map, P->rhs_out, counters);
        CU(cudaMemcpyAsync(&nm, flag + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    if (n > 0) {
        kp_col_counts<<<gn, kBlock, 0, s>>>(n, P->cs, P->ri, P->v, row_act, col_act, tol, cc);
        inclusive_scan(ctx, cc, n, scan_tmp, MC_KERNEL_OTHER);
        kp_flag_active<<<gn, kBlock, 0, s>>>(n, col_act, flag);
        inclusive_scan(ctx, flag, n, scan_tmp, MC_KERNEL_OTHER);
        kp_compact_cols<<<gn, kBlock, 0, s>>>(n, P->cs, P->ri, P->v, row_act, col_act, tol, flag, cc, new_row, P->obj,
                                              P->cs_out, P->ri_out, P->v_out, P->obj_out, P->col_map);
        CU(cudaMemcpyAsync(&nc, flag + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(&nz, cc + (n - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    CU(cudaMemcpyAsync(&hb, counters, sizeof(int), cudaMemcpyDeviceToHost, s));
    // objective offset: obj[j] * fixed of every fixed variable, in stack order (presolve.cpp:162)
    std::vector<int> hk((size_t)h.rec);
    std::vector<double> hv((size_t)h.rec), hv2((size_t)h.rec);
    if (h.rec > 0) {
        CU(cudaMemcpyAsync(hk.data(), R.kind, sizeof(int) * h.rec, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(hv.data(), R.value, sizeof(double) * h.rec, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(hv2.data(), R.value2, sizeof(double) * h.rec, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    TRY(ctx.launch_check("presolve compaction"));
    double offset = lp->objective_offset;
    for (long long t = 0; t < h.rec; ++t)
        if (hk[(size_t)t] == MC_RECORD_FIXED_VARIABLE) {
            const volatile double prod = hv2[(size_t)t] * hv[(size_t)t];  // rounded before the add
            offset += prod;
        }
    I.presolved_rows = nm;
    I.presolved_cols = nc;
    I.presolved_nnz = nz;
    I.objective_offset = offset;
    std::snprintf(I.message, sizeof I.message, "presolve complete");
    // the reduced model's validate() (presolve.cpp:211-213)
    if (nm > 0 && nc > 0) {
        if (hb) return set_error(MC_ERR_INVALID_ARGUMENT, "canonical rhs non-finite");
        if (!std::isfinite(offset)) return set_error(MC_ERR_INVALID_ARGUMENT, "canonical offset non-finite");
    }
    return MC_OK;
}

int presolve_run(Ctx& ctx, const mc_canonical_lp* lp, const mc_presolve_options* o, mc_presolve** out) {
    const double t0 = now_ms();
    if (!out) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve: null result pointer");
    *out = nullptr;
    if (!lp || !o) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve: null argument");
    const int m = lp->num_rows, n = lp->num_cols;
    const long long nnz = lp->nnz;
    if (m < 0 || n < 0 || nnz < 0 || !lp->col_start || (m > 0 && !lp->rhs) || (n > 0 && !lp->objective) ||
        (nnz > 0 && (!lp->row_index || !lp->value)))
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve: malformed canonical model");
    if (nnz >= INT_MAX || (long long)m + n >= INT_MAX / 2)
        return set_error(MC_ERR_RESOURCE_LIMIT, "presolve: model beyond the int32 index range");
    if (!std::isfinite(lp->objective_offset)) return set_error(MC_ERR_INVALID_ARGUMENT, "canonical offset non-finite");
    if (o->max_passes < 0 || !std::isfinite(o->feasibility_tolerance) || !std::isfinite(o->dual_tolerance) ||
        !std::isfinite(o->pivot_tolerance))
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve: invalid options");
    ctx.drop_session();
    mc_presolve* P = new mc_presolve();
    P->device = ctx.device;
    P->m = m;
    P->n = n;
    P->nnz = nnz;
    P->offset = lp->objective_offset;
    const int rc = presolve_body(ctx, lp, o, P);
    if (rc != MC_OK) {
        ps_free(P);
        return rc;
    }
    P->info.presolve_ms = now_ms() - t0;
    *out = P;
    return MC_OK;
}

int presolve_load(Ctx& ctx, const mc_canonical_lp* lp, long long nrec, const int* kind, const long long* index,
                  const long long* variable, const double* value, const double* value2, long long pm,
                  const long long* row_map, long long pn, const long long* col_map, mc_presolve** out) {
    if (!out) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve load: null result pointer");
    *out = nullptr;
    if (!lp || nrec < 0 || pm < 0 || pn < 0 || (nrec > 0 && (!kind || !index || !variable || !value || !value2)) ||
        (pm > 0 && !row_map) || (pn > 0 && !col_map))
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve load: null argument");
    const int m = lp->num_rows, n = lp->num_cols;
    if (m < 0 || n < 0 || lp->nnz < 0 || !lp->col_start || (n > 0 && !lp->objective) ||
        (lp->nnz > 0 && (!lp->row_index || !lp->value)))
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve load: malformed canonical model");
    if (nrec > (long long)m + n || pm > m || pn > n)
        return set_error(MC_ERR_INVALID_ARGUMENT, "presolve load: more records or map entries than lines");
    // the records and maps index the model's lines (postsolve reads through them)
    for (long long t = 0; t < nrec; ++t) {
        const long long i = index[t];
        switch (kind[t]) {
            case MC_RECORD_EMPTY_ROW:
                if (i < 0 || i >= m) return set_error(MC_ERR_INVALID_ARGUMENT, "record %lld: row out of range", t);
                break;
            case MC_RECORD_EMPTY_COLUMN:
            case MC_RECORD_FIXED_VARIABLE:
                if (i < 0 || i >= n) return set_error(MC_ERR_INVALID_ARGUMENT, "record %lld: column out of range", t);
                break;
            case MC_RECORD_ROW_SINGLETON:
                if (i < 0 || i >= m || variable[t] < 0 || variable[t] >= n || value[t] == 0.0)
                    return set_error(MC_ERR_INVALID_ARGUMENT, "record %lld: bad row singleton", t);
                break;
            default: return set_error(MC_ERR_INVALID_ARGUMENT, "record %lld: unknown kind %d", t, kind[t]);
        }
    }
    for (long long q = 0; q < pm; ++q)
        if (row_map[q] < 0 || row_map[q] >= m) return set_error(MC_ERR_INVALID_ARGUMENT, "row map out of range");
    for (long long q = 0; q < pn; ++q)
        if (col_map[q] < 0 || col_map[q] >= n) return set_error(MC_ERR_INVALID_ARGUMENT, "column map out of range");
    ctx.drop_session();
    cudaStream_t s = ctx.stream;
    mc_presolve* P = new mc_presolve();
    P->device = ctx.device;
    P->m = m;
    P->n = n;
    P->nnz = lp->nnz;
    P->offset = lp->objective_offset;
    const size_t nn = (size_t)n + 1, zz = (size_t)lp->nnz + 1, rr = (size_t)nrec + 1;
    int rc = MC_OK;
    auto own = [&](auto** ptr, size_t count) {
        if (rc == MC_OK) rc = ps_alloc(P, reinterpret_cast<void**>(ptr), count * sizeof(**ptr), s);
    };
    own(&P->cs, nn);
    own(&P->ri, zz);
    own(&P->v, zz);
    own(&P->obj, nn);
    own(&P->row_map, (size_t)pm + 1);
    own(&P->col_map, (size_t)pn + 1);
    own(&P->R.kind, rr);
    own(&P->R.index, rr);
    own(&P->R.variable, rr);
    own(&P->R.value, rr);
    own(&P->R.value2, rr);
    own(&P->R.inc_off, rr);
    own(&P->R.inc_len, rr);
    if (rc == MC_OK) {
        rc = [&]() -> int {
            const cudaMemcpyKind k = cudaMemcpyDefault;
            CU(cudaMemcpyAsync(P->cs, lp->col_start, sizeof(int) * nn, k, s));
            if (lp->nnz > 0) {
                CU(cudaMemcpyAsync(P->ri, lp->row_index, sizeof(int) * lp->nnz, k, s));
                CU(cudaMemcpyAsync(P->v, lp->value, sizeof(double) * lp->nnz, k, s));
            }
            if (n > 0) CU(cudaMemcpyAsync(P->obj, lp->objective, sizeof(double) * n, k, s));
            if (pm > 0) CU(cudaMemcpyAsync(P->row_map, row_map, sizeof(long long) * pm, k, s));
            if (pn > 0) CU(cudaMemcpyAsync(P->col_map, col_map, sizeof(long long) * pn, k, s));
            if (nrec > 0) {
                CU(cudaMemcpyAsync(P->R.kind, kind, sizeof(int) * nrec, k, s));
                CU(cudaMemcpyAsync(P->R.index, index, sizeof(long long) * nrec, k, s));
                CU(cudaMemcpyAsync(P->R.variable, variable, sizeof(long long) * nrec, k, s));
                CU(cudaMemcpyAsync(P->R.value, value, sizeof(double) * nrec, k, s));
                CU(cudaMemcpyAsync(P->R.value2, value2, sizeof(double) * nrec, k, s));
                CU(cudaMemsetAsync(P->R.inc_len, 0, sizeof(int) * nrec, s));
            }
            CU(cudaStreamSynchronize(s));
            // the column structure postsolve walks (singleton columns), checked like presolve's input
            int* bad = nullptr;
            CU(cudaMallocAsync(reinterpret_cast<void**>(&bad), sizeof(int), s));
            CU(cudaMemsetAsync(bad, 0, sizeof(int), s));
            if (n > 0) k_validate_csc<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, lp->nnz, P->cs, P->ri, P->v, bad);
            int hb = 0;
            CU(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
            CU(cudaFreeAsync(bad, s));
            CU(cudaStreamSynchronize(s));
            TRY(ctx.launch_check("presolve load"));
            if (hb) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve load: invalid canonical CSC (flags %d)", hb);
            return MC_OK;
        }();
    }
    if (rc != MC_OK) {
        cudaStreamSynchronize(s);
        ps_free(P);
        return rc;
    }
    mc_presolve_info& I = P->info;
    I.status = MC_PRESOLVE_OPTIMAL;
    I.original_rows = m;
    I.original_cols = n;
    I.presolved_rows = pm;
    I.presolved_cols = pn;
    I.records = nrec;
    std::snprintf(I.message, sizeof I.message, "loaded");
    *out = P;
    return MC_OK;
}

int postsolve_body(Ctx& ctx, const mc_presolve* P, const double* rx, long long rx_len, const double* ry,
                   long long ry_len, double* x_out, double* y_out, double* objective) {
    cudaStream_t s = ctx.stream;
    const int m = P->m, n = P->n;
    const mc_presolve_info& I = P->info;
    PsScratch S(s, ctx.device);
    double *x, *y, *drx, *dry, *pi_in, *pi_out;
    int *pos, *sing = nullptr, *counters;
    unsigned char *done, *now_done;
    DD* parts;
    const int gpart = 256;
    S.get(&x, (size_t)n + 1);
    S.get(&y, (size_t)m + 1);
    S.get(&drx, (size_t)rx_len + 1);
    S.get(&dry, (size_t)ry_len + 1);
    S.get(&pi_in, (size_t)m + 1);
    S.get(&pi_out, (size_t)m + 1);
    S.get(&pos, (size_t)m + 1);
    S.get(&done, (size_t)m + 1);
    S.get(&now_done, (size_t)m + 1);
    S.get(&counters, 4);
    S.get(&parts, gpart);
    TRY(S.rc);
    if ((rx_len > 0 && cudaMemcpyAsync(drx, rx, sizeof(double) * rx_len, cudaMemcpyDefault, s) != cudaSuccess) ||
        (ry_len > 0 && cudaMemcpyAsync(dry, ry, sizeof(double) * ry_len, cudaMemcpyDefault, s) != cudaSuccess)) {
        cudaGetLastError();
        return set_error(MC_ERR_INVALID_ARGUMENT, "postsolve: cannot read the reduced solution");
    }
    const int g = blocks_for(ctx, std::max(std::max(m, n), 1), kBlock);
    // presolve.cpp:257-272: zeros, then the reduced solution through the maps
    kp_post_zero<<<g, kBlock, 0, s>>>(m, n, x, y);
    kp_post_place<<<g, kBlock, 0, s>>>(I.presolved_rows, I.presolved_cols, P->row_map, P->col_map, drx, rx_len, dry,
                                       ry_len, x, y);
    CU(cudaMemsetAsync(pos, 0xff, sizeof(int) * ((size_t)m + 1), s));  // -1: not a singleton row
    CU(cudaMemsetAsync(done, 0, (size_t)m + 1, s));
    CU(cudaMemsetAsync(now_done, 0, (size_t)m + 1, s));
    CU(cudaMemsetAsync(pi_in, 0, sizeof(double) * ((size_t)m + 1), s));
    const long long nrec = I.records;
    if (nrec > 0) kp_post_records<<<blocks_for(ctx, nrec, kBlock), kBlock, 0, s>>>(nrec, P->R, x, pos);
    // the singleton records' stack positions
    std::vector<int> hk((size_t)nrec);
    if (nrec > 0) CU(cudaMemcpyAsync(hk.data(), P->R.kind, sizeof(int) * nrec, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.launch_check("postsolve scatter"));
    std::vector<int> hs;
    for (long long t = 0; t < nrec; ++t)
        if (hk[(size_t)t] == MC_RECORD_ROW_SINGLETON) hs.push_back((int)t);
    const int ns = (int)hs.size();
    if (ns > 0) {
        S.get(&sing, (size_t)ns);
        TRY(S.rc);
        CU(cudaMemcpyAsync(sing, hs.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, s));
        const int gs = blocks_for(ctx, ns, kBlock);
        int left = ns;
        while (left > 0) {
            CU(cudaMemsetAsync(counters, 0, sizeof(int) * 2, s));
            kp_post_wave<<<gs, kBlock, 0, s>>>(ns, sing, P->R, P->cs, P->ri, P->v, P->obj, pos, done, y, pi_in,
                                                pi_out, now_done, counters);
            kp_post_mark<<<gs, kBlock, 0, s>>>(ns, sing, P->R, now_done, done, pi_out, pi_in);
            int hc[2] = {0, 0};
            CU(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            TRY(ctx.launch_check("postsolve wave"));
            if (hc[1]) return set_error(MC_ERR_INVALID_ARGUMENT, "non-finite dual multiplier in postsolve");
            if (hc[0] >= left) return set_error(MC_ERR_INTERNAL, "postsolve: no singleton record ready");
            left = hc[0];
        }
        kp_post_duals<<<gs, kBlock, 0, s>>>(ns, sing, P->R, pi_in, y);
    }
    // presolve.cpp:303-308
    kp_post_objective<<<gpart, kBlock, 0, s>>>(n, P->obj, x, parts);
    std::vector<DD> hp(gpart);
    CU(cudaMemcpyAsync(hp.data(), parts, sizeof(DD) * gpart, cudaMemcpyDeviceToHost, s));
    if (n > 0) CU(cudaMemcpyAsync(x_out, x, sizeof(double) * n, cudaMemcpyDefault, s));
    if (m > 0) CU(cudaMemcpyAsync(y_out, y, sizeof(double) * m, cudaMemcpyDefault, s));
    CU(cudaStreamSynchronize(s));
    TRY(ctx.launch_check("postsolve"));
    DD tot{P->offset, 0.0};
    for (const DD& d : hp) tot = dd_add(tot, d);
    *objective = tot.hi + tot.lo;
    if (!std::isfinite(*objective)) return set_error(MC_ERR_INVALID_ARGUMENT, "non-finite objective in postsolve");
    return MC_OK;
}

int postsolve_run(Ctx& ctx, const mc_presolve* P, const double* rx, long long rx_len, const double* ry,
                  long long ry_len, double* x_out, double* y_out, double* objective) {
    if (!P || !objective || (P->n > 0 && !x_out) || (P->m > 0 && !y_out) || rx_len < 0 || ry_len < 0 ||
        (rx_len > 0 && !rx) || (ry_len > 0 && !ry))
        return set_error(MC_ERR_INVALID_ARGUMENT, "postsolve: null argument");
    if (P->device != ctx.device) return set_error(MC_ERR_INVALID_ARGUMENT, "postsolve: presolve of another device");
    ctx.drop_session();
    return postsolve_body(ctx, P, rx, rx_len, ry, ry_len, x_out, y_out, objective);
}

}  // namespace mc

// ------------------------------------------------------------------ C ABI
extern "C" void mc_presolve_default_options(mc_presolve_options* o) {
    if (!o) return;
    o->max_passes = 5;  // presolve.hpp:12-17
    o->feasibility_tolerance = 1e-9;
    o->dual_tolerance = 1e-9;
    o->pivot_tolerance = 1e-12;
}

extern "C" int mc_presolve_run(mc_pdlp_ctx* c, const mc_canonical_lp* lp, const mc_presolve_options* options,
                               mc_presolve** out) {
    using namespace mc;
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return presolve_run(*ctx, lp, options, out);
}

extern "C" int mc_presolve_get_info(const mc_presolve* p, mc_presolve_info* info) {
    if (!p || !info) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "presolve or info is NULL");
    *info = p->info;
    return MC_OK;
}

namespace mc {
// copies `count` elements of a presolve result to a caller buffer (host or device)
template <class T>
int ps_copy(const mc_presolve* p, T* dst, const T* src, long long count) {
    if (!dst || count <= 0) return MC_OK;
    DeviceGuard guard(p->device);
    CU(cudaMemcpy(dst, src, sizeof(T) * (size_t)count, cudaMemcpyDefault));
    return MC_OK;
}
}  // namespace mc

extern "C" int mc_presolve_get_model(const mc_presolve* p, int32_t* col_start, int32_t* row_index, double* value,
                                     double* rhs, double* objective) {
    using namespace mc;
    if (!p) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve is NULL");
    const mc_presolve_info& I = p->info;
    TRY(ps_copy(p, col_start, p->cs_out, I.presolved_cols + 1));
    TRY(ps_copy(p, row_index, p->ri_out, I.presolved_nnz));
    TRY(ps_copy(p, value, p->v_out, I.presolved_nnz));
    TRY(ps_copy(p, rhs, p->rhs_out, I.presolved_rows));
    TRY(ps_copy(p, objective, p->obj_out, I.presolved_cols));
    return MC_OK;
}

extern "C" int mc_presolve_get_maps(const mc_presolve* p, int64_t* row_map, int64_t* col_map) {
    using namespace mc;
    if (!p) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve is NULL");
    static_assert(sizeof(int64_t) == sizeof(long long), "int64_t is long long");
    TRY(ps_copy(p, reinterpret_cast<long long*>(row_map), p->row_map, p->info.presolved_rows));
    TRY(ps_copy(p, reinterpret_cast<long long*>(col_map), p->col_map, p->info.presolved_cols));
    return MC_OK;
}

extern "C" int mc_presolve_get_records(const mc_presolve* p, int32_t* kind, int64_t* index, int64_t* variable,
                                       double* value, double* value2, int64_t* incident_start, int64_t* incident_row,
                                       double* incident_coefficient) {
    using namespace mc;
    if (!p) return set_error(MC_ERR_INVALID_ARGUMENT, "presolve is NULL");
    const long long nr = p->info.records, ni = p->info.incident_entries;
    TRY(ps_copy(p, kind, p->R.kind, nr));
    TRY(ps_copy(p, reinterpret_cast<long long*>(index), p->R.index, nr));
    TRY(ps_copy(p, reinterpret_cast<long long*>(variable), p->R.variable, nr));
    TRY(ps_copy(p, value, p->R.value, nr));
    TRY(ps_copy(p, value2, p->R.value2, nr));
    TRY(ps_copy(p, reinterpret_cast<long long*>(incident_row), p->R.inc_row, ni));
    TRY(ps_copy(p, incident_coefficient, p->R.inc_coef, ni));
    if (incident_start) {  // from each record's (offset, length); records without a list are empty
        std::vector<long long> off((size_t)nr);
        std::vector<int> len((size_t)nr);
        TRY(ps_copy(p, off.data(), p->R.inc_off, nr));
        TRY(ps_copy(p, len.data(), p->R.inc_len, nr));
        std::vector<long long> st((size_t)nr + 1);
        st[0] = 0;
        for (long long t = 0; t < nr; ++t) {
            st[(size_t)t + 1] = st[(size_t)t] + len[(size_t)t];
            if (len[(size_t)t] > 0 && off[(size_t)t] != st[(size_t)t])
                return set_error(MC_ERR_INTERNAL, "presolve: incident lists out of stack order");
        }
        TRY(ps_copy(p, reinterpret_cast<long long*>(incident_start), (const long long*)st.data(), nr + 1));
    }
    return MC_OK;
}

extern "C" int mc_postsolve(mc_pdlp_ctx* c, const mc_presolve* p, const double* reduced_primal, int64_t reduced_cols,
                            const double* reduced_dual, int64_t reduced_rows, double* primal, double* dual,
                            double* objective) {
    using namespace mc;
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return postsolve_run(*ctx, p, reduced_primal, reduced_cols, reduced_dual, reduced_rows, primal, dual, objective);
}

extern "C" void mc_presolve_free(mc_presolve* p) { mc::ps_free(p); }

extern "C" int mc_presolve_load(mc_pdlp_ctx* c, const mc_canonical_lp* original, int64_t records,
                                const int32_t* kind, const int64_t* index, const int64_t* variable,
                                const double* value, const double* value2, int64_t presolved_rows,
                                const int64_t* row_map, int64_t presolved_cols, const int64_t* col_map,
                                mc_presolve** out) {
    using namespace mc;
    Ctx* ctx = reinterpret_cast<Ctx*>(c);
    if (!ctx) return set_error(MC_ERR_INVALID_ARGUMENT, "context is NULL");
    DeviceGuard guard(ctx->device);
    return presolve_load(*ctx, original, records, kind, reinterpret_cast<const long long*>(index),
                         reinterpret_cast<const long long*>(variable), value, value2, presolved_rows,
                         reinterpret_cast<const long long*>(row_map), presolved_cols,
                         reinterpret_cast<const long long*>(col_map), out);
}
