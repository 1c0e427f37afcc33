// Tile-staged SpMV kernels: one thread per line (row of CSR, column of CSC),
// the matrix streamed through shared memory.
//
// The lines are cut into tiles of about kStageChunk nonzeros (boundaries
// precomputed once per solve by k_tile_bounds), so every tile carries the same
// amount of matrix data whatever the line lengths.  A tile's slice of the
// index and value arrays -- one contiguous byte range, 16-byte aligned by
// widening it to whole 4-entry groups -- is copied into shared memory with
// cp.async (16-byte, L2-only, evict-first), double buffered: the copy of the
// next tile is in flight while the threads gather and reduce the current one.
// The HBM stream is thus fully coalesced and decoupled from the gathers, and
// every thread has all of its line's column indices at hand to issue its
// gathers back to back.
//
// Each line is summed sequentially in storage order with separate multiply
// and add: the same operations in the same order as the reference's
// spmv / spmv_t (src/lp/first_order/pdlp.cpp:22-44), so A x and A^T y are
// bit-identical to the reference's.
//
// A tile whose slice exceeds the buffer (a line longer than the slack) is
// processed straight from global memory, with the same arithmetic.
#pragma once

#include "common.cuh"
#include "iter_kernels.cuh"

namespace mc {

// entries per buffer (2 buffers per block, 96 KB of shared memory either way)
template <class T> struct StageCap { static constexpr int value = 4096; };
template <> struct StageCap<float> { static constexpr int value = 6144; };
// nonzeros per tile: the buffer minus slack for the line that straddles the
// tile's end (lines up to 256 long always fit)
template <class T> constexpr int stage_chunk() { return StageCap<T>::value - 256; }

template <class T>
constexpr size_t staged_smem_bytes() {
    return (size_t)2 * StageCap<T>::value * (sizeof(int) + sizeof(T));
}

// Tile t = lines [bounds[t], bounds[t+1]): bounds[t] is the first line whose
// entries start at or after t * chunk.  Lines are listed in one tile each.
__global__ void k_tile_bounds(int lines, const int* __restrict__ start, int chunk, int ntiles,
                              int* __restrict__ bounds) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += gridDim.x * blockDim.x) {
        if (t == ntiles) {
            bounds[t] = lines;
            continue;
        }
        const long long target = (long long)t * chunk;
        int lo = 0, hi = lines;  // first i in [0, lines] with start[i] >= target
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((long long)start[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        bounds[t] = (t == 0) ? 0 : lo;
    }
}

__device__ __forceinline__ unsigned long long policy_stream() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src, unsigned long long pol) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst), "l"(gmem_src),
                 "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Sequential dot of a line: sum_{p in [b,e)} val[p] * v[idx[p]], multiply then
// add in storage order; four gathers in flight per step.
template <class T>
__device__ __forceinline__ T seq_dot(const int* idx, const T* val, int b, int e, const T* __restrict__ v,
                                     unsigned long long pol) {
    T s = T(0);
    int p = b;
    for (; p + 4 <= e; p += 4) {
        const int i0 = idx[p], i1 = idx[p + 1], i2 = idx[p + 2], i3 = idx[p + 3];
        const T g0 = ld_keep(v + i0, pol), g1 = ld_keep(v + i1, pol), g2 = ld_keep(v + i2, pol),
                g3 = ld_keep(v + i3, pol);
        s = add_rn(s, mul_rn(val[p], g0));
        s = add_rn(s, mul_rn(val[p + 1], g1));
        s = add_rn(s, mul_rn(val[p + 2], g2));
        s = add_rn(s, mul_rn(val[p + 3], g3));
    }
    for (; p < e; ++p) s = add_rn(s, mul_rn(val[p], ld_keep(v + idx[p], pol)));
    return s;
}

// Same, two vectors at once (A x-bar and A dx).
template <class T>
__device__ __forceinline__ void seq_dot2(const int* idx, const T* val, int b, int e, const T* __restrict__ vw,
                                         unsigned long long pol, T& sv, T& sw) {
    sv = T(0);
    sw = T(0);
    int p = b;
    for (; p + 2 <= e; p += 2) {
        const int i0 = idx[p], i1 = idx[p + 1];
        T v0, w0, v1, w1;
        ld_keep2(vw + 2LL * i0, pol, v0, w0);
        ld_keep2(vw + 2LL * i1, pol, v1, w1);
        sv = add_rn(sv, mul_rn(val[p], v0));
        sw = add_rn(sw, mul_rn(val[p], w0));
        sv = add_rn(sv, mul_rn(val[p + 1], v1));
        sw = add_rn(sw, mul_rn(val[p + 1], w1));
    }
    if (p < e) {
        T v0, w0;
        ld_keep2(vw + 2LL * idx[p], pol, v0, w0);
        sv = add_rn(sv, mul_rn(val[p], v0));
        sw = add_rn(sw, mul_rn(val[p], w0));
    }
}

// The tile loop.  `f(line, idx, val, b, e)` is called once per line of the
// block's tiles with the line's entries at idx[b..e), val[b..e) (shared
// memory when staged, global otherwise).  Every thread of the block runs the
// same number of loop trips and barriers.
template <class T, class F>
__device__ __forceinline__ void stream_lines(const int* __restrict__ bounds, int ntiles,
                                             const int* __restrict__ start, const int* __restrict__ idx,
                                             const T* __restrict__ val, F&& f) {
    constexpr int CAP = StageCap<T>::value;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int* sidx = reinterpret_cast<int*>(smem_raw);
    T* sval = reinterpret_cast<T*>(smem_raw + (size_t)2 * CAP * sizeof(int));
    constexpr int VPC = 16 / sizeof(T);  // values per 16-byte chunk
    const unsigned long long pol = policy_stream();

    // issue the copies of tile t into buffer `buf`; false if not staged
    auto issue = [&](int t, int buf) -> bool {
        if (t >= ntiles) return false;
        const int b = __ldg(start + __ldg(bounds + t)), e = __ldg(start + __ldg(bounds + t + 1));
        const int ba = b & ~3, ea = (e + 3) & ~3;
        if (ea - ba > CAP) return false;
        const int ichunks = (ea - ba) >> 2;
        const int vchunks = (ea - ba) / VPC;
        int* di = sidx + buf * CAP;
        T* dv = sval + buf * CAP;
        for (int c = threadIdx.x; c < ichunks; c += blockDim.x) cp_async16(di + 4 * c, idx + ba + 4 * c, pol);
        for (int c = threadIdx.x; c < vchunks; c += blockDim.x) cp_async16(dv + VPC * c, val + ba + VPC * c, pol);
        return true;
    };

    int tile = blockIdx.x;
    bool staged = issue(tile, 0);
    cp_async_commit();
    for (int q = 0; tile < ntiles; tile += gridDim.x, ++q) {
        const int cur = q & 1;
        const bool staged_next = issue(tile + gridDim.x, cur ^ 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int l0 = __ldg(bounds + tile), l1 = __ldg(bounds + tile + 1);
        const int base = __ldg(start + l0) & ~3;
        for (int line = l0 + threadIdx.x; line < l1; line += blockDim.x) {
            const int b = __ldg(start + line), e = __ldg(start + line + 1);
            if (staged) f(line, sidx + cur * CAP, sval + cur * CAP, b - base, e - base);
            else f(line, idx, val, b, e);
        }
        __syncthreads();
        staged = staged_next;
    }
    cp_async_wait<0>();
}

// Tile boundaries of the two matrix copies (device arrays built at setup).
struct Tiles {
    const int* col_bounds;  // [ncol_tiles + 1]
    const int* row_bounds;  // [nrow_tiles + 1]
    int ncol_tiles, nrow_tiles;
};

// ----------------------------------------------------------------- primal
template <bool STEP, class T>
__global__ void __launch_bounds__(kBlock) k_primal_staged(Iterates<T> P, Tiles Tl, int k) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    const T step = T(st->eta / st->omega);
    const T cnt = T((double)(st->avg_count + k + 1));
    const unsigned long long keep = policy_keep();
    double acc = 0.0;
    stream_lines<T>(Tl.col_bounds, Tl.ncol_tiles, P.csc_start, P.csc_row, P.csc_val,
                    [&](int j, const int* idx, const T* val, int b, int e) {
                        const T aty = seq_dot(idx, val, b, e, P.y, keep);
                        const T cn = ld_stream(P.col_norm + j);
                        const T g = add_rn(ld_stream(P.c + j), aty);
                        const T tau = div_rn(step, cn);
                        const T xo = ld_stream(P.x + j);
                        const T xp = clampv(sub_rn(xo, mul_rn(tau, g)), ld_stream(P.lo + j), ld_stream(P.hi + j));
                        const T d = sub_rn(xp, xo);
                        const T xb = sub_rn(mul_rn(T(2), xp), xo);
                        if (STEP) {
                            st_keep2(P.xdx + 2LL * j, xb, d, keep);
                            acc += __dmul_rn(__dmul_rn((double)cn, (double)d), (double)d);
                        } else {
                            st_keep(P.x_bar + j, xb, keep);
                        }
                        st_stream(P.x + j, xp);
                        const T xa = ld_stream(P.x_avg + j);
                        st_stream(P.x_avg + j, add_rn(xa, div_rn(sub_rn(xp, xa), cnt)));
                    });
    if (STEP) {
        acc = block_reduce(acc, scratch, OpSum());
        if (threadIdx.x == 0) P.partials[SLOT_DX * kMaxPartials + blockIdx.x] = acc;
    }
}

// ------------------------------------------------------------------- dual
template <class T>
__global__ void __launch_bounds__(kBlock) k_dual_staged(Iterates<T> P, Tiles Tl, int k) {
    const DevState* st = P.st;
    if (st->done) return;
    const T sg = T(st->eta * st->omega);
    const T cnt = T((double)(st->avg_count + k + 1));
    const unsigned long long keep = policy_keep();
    stream_lines<T>(Tl.row_bounds, Tl.nrow_tiles, P.csr_start, P.csr_col, P.csr_val,
                    [&](int i, const int* idx, const T* val, int b, int e) {
                        const T ax = seq_dot(idx, val, b, e, P.x_bar, keep);
                        dual_update(P, i, ax, sg, cnt, keep);
                    });
}

// Step-size iteration, part 1 (see k_dual_probe).
template <class T>
__global__ void __launch_bounds__(kBlock) k_dual_probe_staged(Iterates<T> P, Tiles Tl) {
    __shared__ double scratch[32];
    const DevState* st = P.st;
    if (st->done) return;
    const unsigned long long keep = policy_keep();
    double acc = 0.0;
    stream_lines<T>(Tl.row_bounds, Tl.nrow_tiles, P.csr_start, P.csr_col, P.csr_val,
                    [&](int i, const int* idx, const T* val, int b, int e) {
                        T axb, adx;
                        seq_dot2(idx, val, b, e, P.xdx, keep, axb, adx);
                        P.ax_bar[i] = axb;
                        const double a = (double)adx;
                        acc += __ddiv_rn(__dmul_rn(a, a), (double)P.row_norm[i]);
                    });
    acc = block_reduce(acc, scratch, OpSum());
    if (threadIdx.x == 0) P.partials[SLOT_ADX * kMaxPartials + blockIdx.x] = acc;
}

}  // namespace mc
