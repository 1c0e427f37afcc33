// One-time kernels of a solve: input validation, CSC -> CSR transpose,
// Ruiz equilibration, L1 norms and the initial iterate.  All run in FP64;
// none is on the per-iteration path.
#pragma once

#include "common.cuh"

namespace mc {

template <class T>
__global__ void k_fill(T* __restrict__ a, long long n, T v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        a[i] = v;
}

// max row length (for the long-row sort path)
__global__ void k_max_line(int lines, const int* __restrict__ start, int* __restrict__ out) {
    int mx = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lines; i += gridDim.x * blockDim.x)
        mx = max(mx, start[i + 1] - start[i]);
    for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// ---------------------------------------------------------------- validation
// Flags what SparseMatrixCSC::validate rejects (src/model/model.cpp:41-66):
// bad pointers, row index out of range, rows not strictly increasing, zero or
// non-finite values.  Guarding device-resident input keeps every later gather
// in bounds.
__global__ void k_validate_csc(int m, int n, long long nnz, const int* __restrict__ col_start,
                               const int* __restrict__ row_index, const double* __restrict__ value,
                               int* __restrict__ bad) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int b = col_start[j], e = col_start[j + 1];
    if (j == 0 && b != 0) atomicOr(bad, 1);
    if (j == n - 1 && (long long)e != nnz) atomicOr(bad, 1);
    if (b > e || b < 0 || (long long)e > nnz) { atomicOr(bad, 1); return; }
    int prev = -1;
    for (int p = b; p < e; ++p) {
        const int r = row_index[p];
        const double v = value[p];
        if (r < 0 || r >= m) { atomicOr(bad, 2); return; }
        if (r <= prev) { atomicOr(bad, 4); return; }
        if (!isfinite(v) || v == 0.0) { atomicOr(bad, 8); return; }
        prev = r;
    }
}

// ----------------------------------------------------------------- transpose
// counts[r + 1] += 1 for every entry of row r
__global__ void k_count_rows(long long nnz, const int* __restrict__ row_index, int* __restrict__ counts) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nnz;
         p += (long long)gridDim.x * blockDim.x)
        atomicAdd(&counts[row_index[p] + 1], 1);
}

// In-place inclusive scan of int32 in tiles of kScanTile per block; the
// tile totals go to `totals` (one per block).
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int* __restrict__ data, long long n, int* __restrict__ totals) {
    __shared__ int warp_sums[32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int run = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const long long i = base + q;
        run += (i < n) ? data[i] : 0;
        v[q] = run;
    }
    // exclusive scan of per-thread totals across the block
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int t = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, t, off);
        if (lane >= off) t += o;
    }
    if (lane == 31) warp_sums[warp] = t;
    __syncthreads();
    if (warp == 0) {
        int w = warp_sums[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += o;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    const int before = (t - run) + (warp > 0 ? warp_sums[warp - 1] : 0);
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const long long i = base + q;
        if (i < n) data[i] = v[q] + before;
    }
    if (threadIdx.x == kScanThreads - 1) totals[blockIdx.x] = before + run;
}

// adds the scanned total of all previous tiles to every element of a tile
__global__ void k_scan_add(int* __restrict__ data, long long n, const int* __restrict__ scanned_totals) {
    if (blockIdx.x == 0) return;
    const int add = scanned_totals[blockIdx.x - 1];
    const long long base = (long long)blockIdx.x * kScanTile;
    for (int q = threadIdx.x; q < kScanTile; q += blockDim.x) {
        const long long i = base + q;
        if (i < n) data[i] += add;
    }
}

// Unordered scatter of CSC entries into their CSR rows (thread per column).
__global__ void k_scatter_rows(int n, const int* __restrict__ col_start, const int* __restrict__ row_index,
                               const double* __restrict__ value, const int* __restrict__ row_start,
                               int* __restrict__ cursor, int* __restrict__ col_index,
                               double* __restrict__ csr_value) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int p = col_start[j]; p < col_start[j + 1]; ++p) {
        const int r = row_index[p];
        const int pos = row_start[r] + atomicAdd(&cursor[r], 1);
        col_index[pos] = j;
        csr_value[pos] = value[p];
    }
}

constexpr int kShortRow = 32;     // rows up to this length: thread-level insertion sort
constexpr int kSmemSortRow = 4096;  // rows up to this length: shared-memory bitonic sort

// Sorts short rows by column (insertion sort, thread per row) and lists the
// long rows for the block-level sort.
__global__ void k_sort_short_rows(int m, const int* __restrict__ row_start, int* __restrict__ col_index,
                                  double* __restrict__ value, int* __restrict__ long_rows,
                                  int* __restrict__ long_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int b = row_start[i], e = row_start[i + 1];
    if (e - b > kShortRow) {
        long_rows[atomicAdd(long_count, 1)] = i;
        return;
    }
    for (int p = b + 1; p < e; ++p) {
        const int key = col_index[p];
        const double v = value[p];
        int q = p - 1;
        while (q >= b && col_index[q] > key) {
            col_index[q + 1] = col_index[q];
            value[q + 1] = value[q];
            --q;
        }
        col_index[q + 1] = key;
        value[q + 1] = v;
    }
}

// One block per long row.  Rows up to kSmemSortRow: bitonic sort in shared
// memory.  Longer rows: each element's final slot is its rank (columns are
// distinct within a row), written to scratch and copied back.
__global__ void __launch_bounds__(1024) k_sort_long_rows(const int* __restrict__ long_rows,
                                                         const int* __restrict__ row_start,
                                                         int* __restrict__ col_index,
                                                         double* __restrict__ value,
                                                         int* __restrict__ tmp_col,
                                                         double* __restrict__ tmp_val) {
    extern __shared__ unsigned char smem_raw[];
    const int i = long_rows[blockIdx.x];
    const int b = row_start[i], e = row_start[i + 1];
    const int len = e - b;
    if (len <= kSmemSortRow) {
        int pow2 = 1;
        while (pow2 < len) pow2 <<= 1;
        int* keys = reinterpret_cast<int*>(smem_raw);
        double* vals = reinterpret_cast<double*>(smem_raw + kSmemSortRow * sizeof(int));
        for (int q = threadIdx.x; q < pow2; q += blockDim.x) {
            keys[q] = (q < len) ? col_index[b + q] : 0x7fffffff;
            vals[q] = (q < len) ? value[b + q] : 0.0;
        }
        __syncthreads();
        for (int size = 2; size <= pow2; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int q = threadIdx.x; q < pow2; q += blockDim.x) {
                    const int partner = q ^ stride;
                    if (partner > q) {
                        const bool up = (q & size) == 0;
                        const int a = keys[q], c = keys[partner];
                        if ((a > c) == up) {
                            keys[q] = c;
                            keys[partner] = a;
                            const double tv = vals[q];
                            vals[q] = vals[partner];
                            vals[partner] = tv;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int q = threadIdx.x; q < len; q += blockDim.x) {
            col_index[b + q] = keys[q];
            value[b + q] = vals[q];
        }
    } else {
        for (int q = threadIdx.x; q < len; q += blockDim.x) {
            const int key = col_index[b + q];
            int rank = 0;
            for (int t = 0; t < len; ++t) rank += (col_index[b + t] < key) ? 1 : 0;
            tmp_col[b + rank] = key;
            tmp_val[b + rank] = value[b + q];
        }
        __syncthreads();
        for (int q = threadIdx.x; q < len; q += blockDim.x) {
            col_index[b + q] = tmp_col[b + q];
            value[b + q] = tmp_val[b + q];
        }
    }
}

// ---------------------------------------------------------------------- Ruiz
// equilibrate_model, src/scale/ruiz_scaling.cpp:167-218, one pass split into
// norms (max |a| per column over CSC, per row over CSR), the convergence test
// and the rescaling of both copies.  Maxima are exact in any order, and the
// rescale computes value * (delta_r[i] * delta_c[j]) exactly as :215, so the
// scaled matrix equals the reference's bit for bit.

// norm[j] = max |a| of line j (0 -> 1), err partial = max |1 - norm|
__global__ void k_ruiz_line_max(int lines, const int* __restrict__ start, const double* __restrict__ value,
                                double* __restrict__ norm, double* __restrict__ err_partials,
                                const DevState* __restrict__ st) {
    __shared__ double scratch[32];
    if (st->ruiz_done) return;
    double err = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        double mx = 0.0;
        for (int p = start[j]; p < start[j + 1]; ++p) mx = maxv(mx, fabs(value[p]));
        if (mx == 0.0) mx = 1.0;
        norm[j] = mx;
        err = maxv(err, fabs(1.0 - mx));
    }
    err = block_reduce(err, scratch, OpMax());
    if (threadIdx.x == 0) err_partials[blockIdx.x] = err;
}

// convergence test (:185-197); on success later passes become no-ops
__global__ void k_ruiz_check(const double* __restrict__ row_err, int nrow_parts,
                             const double* __restrict__ col_err, int ncol_parts, double tolerance,
                             DevState* __restrict__ st) {
    __shared__ double scratch[32];
    if (st->ruiz_done) return;
    const double r = reduce_partials(row_err, nrow_parts, scratch, OpMax());
    const double c = reduce_partials(col_err, ncol_parts, scratch, OpMax());
    if (threadIdx.x == 0) {
        if (r < tolerance && c < tolerance) st->ruiz_done = 1;
        else st->ruiz_passes += 1;
    }
}

// delta = 1/sqrt(norm) (stored over norm), scale *= delta  (:199-208)
__global__ void k_ruiz_deltas(int lines, double* __restrict__ norm, double* __restrict__ scale,
                              const DevState* __restrict__ st) {
    if (st->ruiz_done) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        const double d = 1.0 / sqrt(norm[j]);
        norm[j] = d;
        scale[j] *= d;
    }
}

// a_p *= delta_outer[line] * ... for CSC (outer = column) and CSR (outer = row)
// value[p] *= delta_r[r] * delta_c[c]  with the product formed first (:215)
__global__ void k_ruiz_rescale(int lines, const int* __restrict__ start, const int* __restrict__ inner,
                               double* __restrict__ value, const double* __restrict__ delta_outer,
                               const double* __restrict__ delta_inner, int outer_is_row,
                               const DevState* __restrict__ st) {
    if (st->ruiz_done) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        const double dout = delta_outer[j];
        for (int p = start[j]; p < start[j + 1]; ++p) {
            const double din = delta_inner[inner[p]];
            const double f = outer_is_row ? __dmul_rn(dout, din) : __dmul_rn(din, dout);
            value[p] = __dmul_rn(value[p], f);
        }
    }
}

// ------------------------------------------------------------ problem setup
// Column data (:153-159, :168-176, :186-191 and the Ruiz bound/objective
// scaling :238-244).  Writes the scaled c, bounds (sentinel form), the
// original bounds (sentinel form), L1 column norms, the starting x.
// Partials: SLOT_A max|c|, SLOT_B max|c_orig| (residual scale).
__global__ void k_setup_cols(int n, const int* __restrict__ col_start, const double* __restrict__ value,
                             const double* __restrict__ obj_in, const double* __restrict__ lo_in,
                             const double* __restrict__ hi_in, const double* __restrict__ col_scale,
                             const double* __restrict__ warm_x, double obj_sign,
                             double* __restrict__ c, double* __restrict__ lo, double* __restrict__ hi,
                             double* __restrict__ c_orig, double* __restrict__ lo_orig,
                             double* __restrict__ hi_orig, double* __restrict__ col_norm,
                             double* __restrict__ x, double* __restrict__ x_avg,
                             double* __restrict__ partials) {
    __shared__ double scratch[32];
    double cmax = 0.0, comax = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double s = col_scale[j];
        const double inv = 1.0 / s;
        const double l0 = lo_in[j], h0 = hi_in[j];
        const double ls = isfinite(l0) ? __dmul_rn(l0, inv) : l0;
        const double hs = isfinite(h0) ? __dmul_rn(h0, inv) : h0;
        const double lsent = isinf(ls) ? -kBig : ls;
        const double hsent = isinf(hs) ? kBig : hs;
        lo[j] = lsent;
        hi[j] = hsent;
        lo_orig[j] = isinf(l0) ? -kBig : l0;
        hi_orig[j] = isinf(h0) ? kBig : h0;
        const double cj = obj_sign * __dmul_rn(obj_in[j], s);
        c[j] = cj;
        cmax = maxv(cmax, fabs(cj));
        const double co = obj_sign * obj_in[j];
        c_orig[j] = co;
        comax = maxv(comax, fabs(co));
        double nrm = 0.0;
        for (int p = col_start[j]; p < col_start[j + 1]; ++p) nrm += fabs(value[p]);
        col_norm[j] = (nrm < 1e-12) ? 1.0 : nrm;
        const double start = warm_x ? __dmul_rn(warm_x[j], inv) : 0.0;
        const double x0 = clampv(start, lsent, hsent);
        x[j] = x0;
        x_avg[j] = x0;
    }
    cmax = block_reduce(cmax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_A * kMaxPartials + blockIdx.x] = cmax;
    comax = block_reduce(comax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_B * kMaxPartials + blockIdx.x] = comax;
}

// Row data (:160-167, :168-176, Ruiz row-bound scaling :229-236).
// Partial SLOT_C: max finite |b|.
__global__ void k_setup_rows(int m, const int* __restrict__ row_start, const double* __restrict__ value,
                             const double* __restrict__ rlo_in, const double* __restrict__ rhi_in,
                             const double* __restrict__ row_scale, const double* __restrict__ warm_y,
                             double* __restrict__ blo, double* __restrict__ bhi,
                             double* __restrict__ blo_orig, double* __restrict__ bhi_orig,
                             double* __restrict__ row_norm, double* __restrict__ y,
                             double* __restrict__ y_avg, double* __restrict__ partials) {
    __shared__ double scratch[32];
    double bmax = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const double s = row_scale[i];
        const double l0 = rlo_in[i], h0 = rhi_in[i];
        const double ls = isfinite(l0) ? __dmul_rn(l0, s) : l0;
        const double hs = isfinite(h0) ? __dmul_rn(h0, s) : h0;
        const double lsent = isinf(ls) ? -kBig : ls;
        const double hsent = isinf(hs) ? kBig : hs;
        blo[i] = lsent;
        bhi[i] = hsent;
        blo_orig[i] = isinf(l0) ? -kBig : l0;
        bhi_orig[i] = isinf(h0) ? kBig : h0;
        if (fabs(lsent) < 1e299) bmax = maxv(bmax, fabs(lsent));
        if (fabs(hsent) < 1e299) bmax = maxv(bmax, fabs(hsent));
        double nrm = 0.0;
        for (int p = row_start[i]; p < row_start[i + 1]; ++p) nrm += fabs(value[p]);
        row_norm[i] = (nrm < 1e-12) ? 1.0 : nrm;
        const double y0 = warm_y ? __dmul_rn(warm_y[i], 1.0 / s) : 0.0;
        y[i] = y0;
        y_avg[i] = y0;
    }
    bmax = block_reduce(bmax, scratch, OpMax());
    if (threadIdx.x == 0) partials[SLOT_C * kMaxPartials + blockIdx.x] = bmax;
}

// Scalars (:155-159, :165-166, :177-179) and counters (:192-193).
__global__ void k_setup_scalars(const double* __restrict__ partials, int ncol_parts, int nrow_parts,
                                double initial_primal_weight, double step_size_reduction,
                                DevState* __restrict__ st) {
    __shared__ double scratch[32];
    const double cmax = reduce_partials(partials + SLOT_A * kMaxPartials, ncol_parts, scratch, OpMax());
    const double comax = reduce_partials(partials + SLOT_B * kMaxPartials, ncol_parts, scratch, OpMax());
    const double bmax = reduce_partials(partials + SLOT_C * kMaxPartials, nrow_parts, scratch, OpMax());
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
        st->done = 0;
        st->status = 1;  // iteration_limit until proven otherwise
        st->restart_pending = 0;
        st->nonfinite = 0;
    }
}

// Unscaled averages out (pdlp.cpp:76-79): x = x_avg * D_C, y = y_avg * D_R.
__global__ void k_unscale_out(int n, int m, const double* __restrict__ x_avg, const double* __restrict__ y_avg,
                              const double* __restrict__ col_scale, const double* __restrict__ row_scale,
                              double* __restrict__ x_out, double* __restrict__ y_out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
        if (t < n) {
            if (x_out) x_out[t] = __dmul_rn(x_avg[t], col_scale[t]);
        } else {
            const int i = t - n;
            if (y_out) y_out[i] = __dmul_rn(y_avg[i], row_scale[i]);
        }
    }
}

}  // namespace mc
