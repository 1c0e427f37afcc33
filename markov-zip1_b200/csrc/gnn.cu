// Learned warm start: a bipartite message-passing network over an LP's
// constraint/variable graph, trained and run with hand-written FP32 kernels.
//
// Graph: one node per variable j and per constraint i, an edge per nonzero
// a_ij.  Hidden width 64, R rounds (default 3):
//   encoders    hv0 = relu(Fv Wve + bve)            hc0 = relu(Fc Wce + bce)
//   round r     agc = An hv      (An_ij = a_ij / |A_i|_1)
//               hc  = relu(hc Wcs + agc Wcn + bc)
//               agv = Ant hc     (Ant_ji = a_ij / |A_j|_1)
//               hv  = relu(hv Wvs + agv Wvn + bv)
//   readouts    x_j = hv_j . wx + bx                (primal, in units of |b|_inf)
//               y_i = hc_i . wy + by                (dual, in units of |c|_inf)
//               log omega = mean(hv) . uv + mean(hc) . uc + bw
// Loss: mean (x - x*/|b|)^2 + mean (y - y*/|c|)^2 + 0.1 (log omega - log omega*)^2
// over the targets the GPU PDLP produced for the instance.
//
// Features (sign conventions of the engine: +-INFINITY bounds):
//   variable   [c_j/|c|, lo finite, hi finite, lo/|b| (0 if inf), hi/|b| (0 if inf), |A_j|_1 / max]
//   constraint [lo/|b| (0 if inf), hi/|b| (0 if inf), lo finite, hi finite, |A_i|_1 / max]
//
// Weight gradients are reduced in two fixed-order stages (block partials,
// then one pass), so training is run-to-run deterministic.
#include "mc_pdlp.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

namespace mc {
int set_error(int code, const char* fmt, ...);
struct Ctx;
Ctx* aux_ctx_create(int device);
void aux_ctx_destroy(Ctx* c);
int aux_csr(Ctx* c, int m, int n, long long nnz, const int* cs, const int* ri, const double* v, int* rs, int* ci,
            double* rv);
}

namespace {

constexpr int H = 64;
constexpr int FV = 6;
constexpr int FC = 5;
constexpr int kRows = 64;       // rows per block in the weight-gradient kernels
constexpr int kThreads = 256;

#define GCU(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return mc::set_error(e_ == cudaErrorMemoryAllocation ? MC_ERR_OUT_OF_MEMORY : MC_ERR_CUDA, \
                                 "%s: %s", #call, cudaGetErrorString(e_));                          \
    } while (0)

#define GTRY(expr)                    \
    do {                              \
        const int rc_ = (expr);       \
        if (rc_ != MC_OK) return rc_; \
    } while (0)

// ------------------------------------------------------------- parameters
struct Layout {
    int rounds;
    long long Wve, bve, Wce, bce;
    std::vector<long long> Wcs, Wcn, bc, Wvs, Wvn, bv;
    long long wx, bx, wy, by, uv, uc, bw;
    long long total;
    explicit Layout(int R) : rounds(R) {
        long long o = 0;
        auto take = [&](long long k) { const long long at = o; o += k; return at; };
        Wve = take(FV * H); bve = take(H); Wce = take(FC * H); bce = take(H);
        for (int r = 0; r < R; ++r) {
            Wcs.push_back(take(H * H)); Wcn.push_back(take(H * H)); bc.push_back(take(H));
            Wvs.push_back(take(H * H)); Wvn.push_back(take(H * H)); bv.push_back(take(H));
        }
        wx = take(H); bx = take(1); wy = take(H); by = take(1); uv = take(H); uc = take(H); bw = take(1);
        total = o;
    }
};

// ----------------------------------------------------------------- kernels
// Y[N x H] = act(X1[N x K1] W1[K1 x H] + X2[N x K2] W2[K2 x H] + b)
//
// Tiled: a block computes a 64-row tile of Y; the weights (K x 64) and the
// tile's input rows are staged in shared memory once, and each of the 256
// threads accumulates a 4 x 4 register block (rows ty*4.., columns tx*4..),
// so every weight and input value is read from global memory once per tile
// instead of once per output.  Each output sums b, then X1 W1 over k in
// order, then X2 W2 -- the order of the one-thread-per-output form.
constexpr int kTile = 64;
__device__ __forceinline__ void dense_stage(float (*sA)[kTile + 1], float (*sW)[H], const float* __restrict__ A,
                                            int K, const float* __restrict__ W, long long r0, int rows) {
    for (int q = threadIdx.x; q < kTile * kTile; q += blockDim.x) {
        const int rr = q / kTile, kk = q % kTile;
        sA[rr][kk] = (rr < rows && kk < K) ? A[(r0 + rr) * K + kk] : 0.f;
    }
    for (int q = threadIdx.x; q < K * H; q += blockDim.x) sW[q / H][q % H] = W[q];
}

__global__ void __launch_bounds__(kThreads) g_dense_fwd(int N, const float* __restrict__ X1, int K1,
                                                        const float* __restrict__ W1, const float* __restrict__ X2,
                                                        int K2, const float* __restrict__ W2,
                                                        const float* __restrict__ b, float* __restrict__ Y, int relu) {
    __shared__ float sA[kTile][kTile + 1];
    __shared__ __align__(16) float sW[kTile][H];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (long long r0 = (long long)blockIdx.x * kTile; r0 < N; r0 += (long long)gridDim.x * kTile) {
        const int rows = (int)(N - r0 < kTile ? N - r0 : kTile);
        float acc[4][4];
        for (int j = 0; j < 4; ++j) {
            const float bj = b[tx * 4 + j];
            for (int i = 0; i < 4; ++i) acc[i][j] = bj;
        }
        for (int part = 0; part < 2; ++part) {
            const float* X = part ? X2 : X1;
            const float* W = part ? W2 : W1;
            const int K = part ? K2 : K1;
            if (!X) continue;
            __syncthreads();
            dense_stage(sA, sW, X, K, W, r0, rows);
            __syncthreads();
            for (int k = 0; k < K; ++k) {
                const float4 w = *reinterpret_cast<const float4*>(&sW[k][tx * 4]);
                for (int i = 0; i < 4; ++i) {
                    const float x = sA[ty * 4 + i][k];
                    acc[i][0] = fmaf(x, w.x, acc[i][0]);
                    acc[i][1] = fmaf(x, w.y, acc[i][1]);
                    acc[i][2] = fmaf(x, w.z, acc[i][2]);
                    acc[i][3] = fmaf(x, w.w, acc[i][3]);
                }
            }
        }
        for (int i = 0; i < 4; ++i) {
            const int rr = ty * 4 + i;
            if (rr >= rows) continue;
            float* y = Y + (r0 + rr) * H + tx * 4;
            for (int j = 0; j < 4; ++j) y[j] = relu ? fmaxf(acc[i][j], 0.f) : acc[i][j];
        }
    }
}

// dZ = dY * (Y > 0) in place (relu backward)
__global__ void g_relu_bwd(long long count, const float* __restrict__ Y, float* __restrict__ dY) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x)
        if (Y[t] <= 0.f) dY[t] = 0.f;
}

// dX[N x K] (+)= dZ[N x H] W[K x H]^T
//
// Tiled like g_dense_fwd: a 64-row tile of dZ and all of W in shared memory,
// a 4 x 4 register block per thread (rows ty*4.., output columns tx*4..);
// each output sums over c = 0..H-1 in order, as the one-thread-per-output form.
__global__ void __launch_bounds__(kThreads) g_dense_bwd_x(int N, const float* __restrict__ dZ,
                                                          const float* __restrict__ W, int K, float* __restrict__ dX,
                                                          int accumulate) {
    __shared__ float sZ[kTile][H + 1];
    __shared__ float sW[kTile][H + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (int q = threadIdx.x; q < K * H; q += blockDim.x) sW[q / H][q % H] = W[q];
    for (long long r0 = (long long)blockIdx.x * kTile; r0 < N; r0 += (long long)gridDim.x * kTile) {
        const int rows = (int)(N - r0 < kTile ? N - r0 : kTile);
        __syncthreads();
        for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
            const int rr = q / H, cc = q % H;
            sZ[rr][cc] = (rr < rows) ? dZ[(r0 + rr) * H + cc] : 0.f;
        }
        __syncthreads();
        float acc[4][4] = {};
        for (int c = 0; c < H; ++c) {
            float w[4], z[4];
            for (int j = 0; j < 4; ++j) w[j] = (tx * 4 + j < K) ? sW[tx * 4 + j][c] : 0.f;
            for (int i = 0; i < 4; ++i) z[i] = sZ[ty * 4 + i][c];
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(z[i], w[j], acc[i][j]);
        }
        for (int i = 0; i < 4; ++i) {
            const int rr = ty * 4 + i;
            if (rr >= rows) continue;
            for (int j = 0; j < 4; ++j) {
                const int k = tx * 4 + j;
                if (k >= K) continue;
                float* d = dX + (r0 + rr) * K + k;
                *d = accumulate ? *d + acc[i][j] : acc[i][j];
            }
        }
    }
}

// block partials of X^T dZ ([K x H]) and of the column sums of dZ ([H]) over
// kRows rows per block
__global__ void __launch_bounds__(kThreads) g_dense_bwd_w(int N, const float* __restrict__ X, int K,
                                                          const float* __restrict__ dZ,
                                                          float* __restrict__ part_w, float* __restrict__ part_b) {
    __shared__ float sx[kRows * H];
    __shared__ float sz[kRows * H];
    const int r0 = blockIdx.x * kRows;
    const int rows = min(kRows, N - r0);
    for (int q = threadIdx.x; q < kRows * H; q += blockDim.x) {
        const int rr = q / H, cc = q % H;
        sz[q] = (rr < rows) ? dZ[(long long)(r0 + rr) * H + cc] : 0.f;
        sx[q] = (rr < rows && cc < K) ? X[(long long)(r0 + rr) * K + cc] : 0.f;
    }
    __syncthreads();
    float* pw = part_w + (long long)blockIdx.x * K * H;
    for (int q = threadIdx.x; q < K * H; q += blockDim.x) {
        const int k = q / H, c = q % H;
        float acc = 0.f;
        for (int rr = 0; rr < rows; ++rr) acc = fmaf(sx[rr * H + k], sz[rr * H + c], acc);
        pw[q] = acc;
    }
    if (part_b)
        for (int c = threadIdx.x; c < H; c += blockDim.x) {
            float acc = 0.f;
            for (int rr = 0; rr < rows; ++rr) acc += sz[rr * H + c];
            part_b[(long long)blockIdx.x * H + c] = acc;
        }
}

// out[q] += sum over blocks of part[b][q], in block order
__global__ void g_reduce_parts(int blocks, int width, const float* __restrict__ part, float* __restrict__ out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < width; q += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int b = 0; b < blocks; ++b) acc += part[(long long)b * width + q];
        out[q] += acc;
    }
}

// Out[line][:] (+)= sum_p val[p] * s_line[line] * s_idx[idx[p]] * In[idx[p]][:]
// (one warp per line, two feature columns per lane)
__global__ void g_aggregate(int lines, const int* __restrict__ start, const int* __restrict__ idx,
                            const float* __restrict__ val, const float* __restrict__ s_line,
                            const float* __restrict__ s_idx, const float* __restrict__ In,
                            float* __restrict__ Out, int accumulate) {
    const int lane = threadIdx.x & 31;
    for (long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; w < lines;
         w += ((long long)gridDim.x * blockDim.x) >> 5) {
        float a0 = 0.f, a1 = 0.f;
        const float sl = s_line ? s_line[w] : 1.f;
        for (int p = start[w]; p < start[w + 1]; ++p) {
            const int j = idx[p];
            const float wgt = val[p] * sl * (s_idx ? s_idx[j] : 1.f);
            a0 = fmaf(wgt, In[(long long)j * H + lane], a0);
            a1 = fmaf(wgt, In[(long long)j * H + 32 + lane], a1);
        }
        float* o = Out + w * H;
        if (accumulate) {
            o[lane] += a0;
            o[32 + lane] += a1;
        } else {
            o[lane] = a0;
            o[32 + lane] = a1;
        }
    }
}

// out[r] = X[r] . w + b
__global__ void g_readout(int N, const float* __restrict__ X, const float* __restrict__ w, const float* __restrict__ b,
                          float* __restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        float acc = b[0];
        for (int c = 0; c < H; ++c) acc = fmaf(X[(long long)r * H + c], w[c], acc);
        out[r] = acc;
    }
}

// column means of X [N x H] -> out[H], in two fixed-order stages: each
// block sums a contiguous row range (4 row groups of H columns, combined in
// order), then one block adds the block sums in block order
constexpr int kMeanBlocks = 512;
__global__ void g_col_sum_parts(int N, const float* __restrict__ X, double* __restrict__ parts) {
    __shared__ double sh[kThreads];
    const int c = threadIdx.x % H, grp = threadIdx.x / H, ngrp = kThreads / H;
    const long long per = ((long long)N + gridDim.x - 1) / gridDim.x;
    const long long r0 = blockIdx.x * per, r1 = min((long long)N, r0 + per);
    double acc = 0.0;
    for (long long r = r0 + grp; r < r1; r += ngrp) acc += X[r * H + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (grp == 0) {
        double t = sh[c];
        for (int q = 1; q < ngrp; ++q) t += sh[q * H + c];
        parts[(long long)blockIdx.x * H + c] = t;
    }
}

__global__ void g_col_mean(int N, int nparts, const double* __restrict__ parts, float* __restrict__ out) {
    for (int c = threadIdx.x; c < H; c += blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nparts; ++b) acc += parts[(long long)b * H + c];
        out[c] = (float)(acc / (N > 0 ? N : 1));
    }
}

// squared-error terms and d pred = 2 (pred - t) / N; partial sums per block
__global__ void g_mse(int N, const float* __restrict__ pred, const float* __restrict__ target,
                      float* __restrict__ dpred, double* __restrict__ part) {
    __shared__ double red[kThreads / 32];
    double acc = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
        const float e = pred[r] - target[r];
        acc += (double)e * e;
        dpred[r] = 2.f * e / (float)N;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
        part[blockIdx.x] = s;
    }
}

// dX[r][c] (+)= d[r] * w[c] (+ extra[c])
__global__ void g_outer_add(int N, const float* __restrict__ d, const float* __restrict__ w,
                            const float* __restrict__ extra, float* __restrict__ dX, int accumulate) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)N * H;
         t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / H;
        const int c = (int)(t % H);
        const float v = (d ? d[r] * w[c] : 0.f) + (extra ? extra[c] : 0.f);
        dX[t] = accumulate ? dX[t] + v : v;
    }
}

// block partials of sum_r d[r] X[r][:] and of sum_r d[r]
__global__ void __launch_bounds__(kThreads) g_readout_bwd(int N, const float* __restrict__ X,
                                                          const float* __restrict__ d, float* __restrict__ part_w,
                                                          float* __restrict__ part_b) {
    const int r0 = blockIdx.x * kRows;
    const int rows = min(kRows, N - r0);
    for (int c = threadIdx.x; c < H; c += blockDim.x) {
        float acc = 0.f;
        for (int rr = 0; rr < rows; ++rr) acc = fmaf(d[r0 + rr], X[(long long)(r0 + rr) * H + c], acc);
        part_w[(long long)blockIdx.x * H + c] = acc;
    }
    if (threadIdx.x == 0) {
        float acc = 0.f;
        for (int rr = 0; rr < rows; ++rr) acc += d[r0 + rr];
        part_b[blockIdx.x] = acc;
    }
}

__global__ void g_adam(long long count, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float a = b1 * m1[t] + (1.f - b1) * gt;
        const float v = b2 * m2[t] + (1.f - b2) * gt * gt;
        m1[t] = a;
        m2[t] = v;
        p[t] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
    }
}

// ------------------------------------------------------------------ host
int grid_of(long long work) {
    long long b = (work + kThreads - 1) / kThreads;
    if (b > 4096) b = 4096;
    return b < 1 ? 1 : (int)b;
}

// blocks of the tiled dense kernels: one per 64-row tile, at most four waves' worth
int tile_grid(long long rows) {
    long long b = (rows + kTile - 1) / kTile;
    if (b > 148 * 8) b = 148 * 8;
    return b < 1 ? 1 : (int)b;
}

// One instance on the device: graph, features, activations, gradients.
// A stream-ordered memory pool per device for instance buffers: freed blocks
// stay reserved (up to 2 GiB) for the next instance, so that a call on a large
// LP does not map and unmap its buffers every time.  Lives until exit; where
// one cannot be made, the device's default pool is used.
cudaMemPool_t instance_pool(int device) {
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
        unsigned long long keep = 2ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pools[device] = pool;
    return pool;
}

// Buffers of one instance, on the network's stream; freed (stream-ordered)
// when the instance goes away.
struct Instance {
    int m = 0, n = 0;
    long long nnz = 0;
    int *cs = nullptr, *ri = nullptr, *rs = nullptr, *ci = nullptr;
    float *cv = nullptr, *rv = nullptr, *rinv = nullptr, *cinv = nullptr;
    float *Fv = nullptr, *Fc = nullptr;
    double bscale = 1.0, cscale = 1.0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;
    Instance(int dev, cudaStream_t s) : device(dev), stream(s) {}
    ~Instance() {
        for (void* p : owned) cudaFreeAsync(p, stream);
    }
    template <class T>
    int alloc(T** p, long long count) {
        void* q = nullptr;
        const size_t bytes = sizeof(T) * (size_t)std::max<long long>(count, 1);
        const cudaMemPool_t pool = instance_pool(device);
        GCU(pool ? cudaMallocFromPoolAsync(&q, bytes, pool, stream) : cudaMallocAsync(&q, bytes, stream));
        owned.push_back(q);
        *p = static_cast<T*>(q);
        return MC_OK;
    }
};

}  // namespace

struct mc_gnn {
    int device = 0;
    int rounds = 3;
    Layout L{3};
    float* params = nullptr;
    float* grads = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    long long step = 0;
    cudaStream_t stream = nullptr;
    // activations of the last forward pass
    std::vector<float*> hv, hc, agv, agc;  // hv[0..R], hc[0..R], agv[1..R], agc[1..R]
    float *px = nullptr, *py = nullptr, *mv = nullptr, *mcm = nullptr, *logw = nullptr;
    float *dx = nullptr, *dy = nullptr, *tx = nullptr, *ty = nullptr;
    float *dhv = nullptr, *dhc = nullptr, *dhv2 = nullptr, *dhc2 = nullptr, *dag = nullptr;
    float *part = nullptr;
    double* dpart = nullptr;
    double* mpart = nullptr;  // block sums of the readout's column means
    long long cap_n = -1, cap_m = -1;
    std::vector<void*> ws;
    mc::Ctx* aux = nullptr;  // the engine's transpose, for large instances
    ~mc_gnn() {
        if (device >= 0) cudaSetDevice(device);
        if (aux) mc::aux_ctx_destroy(aux);
        for (void* p : ws) cudaFree(p);
        cudaFree(params);
        cudaFree(grads);
        cudaFree(m1);
        cudaFree(m2);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int reserve_ws(mc_gnn* g, int n, int m) {
    if (n <= g->cap_n && m <= g->cap_m) return MC_OK;
    for (void* p : g->ws) cudaFree(p);
    g->ws.clear();
    g->hv.assign(g->rounds + 1, nullptr);
    g->hc.assign(g->rounds + 1, nullptr);
    g->agv.assign(g->rounds + 1, nullptr);
    g->agc.assign(g->rounds + 1, nullptr);
    auto get = [&](float** p, long long count) -> int {
        void* q = nullptr;
        GCU(cudaMalloc(&q, sizeof(float) * (size_t)std::max<long long>(count, 1)));
        g->ws.push_back(q);
        *p = static_cast<float*>(q);
        return MC_OK;
    };
    const long long nH = (long long)n * H, mH = (long long)m * H;
    for (int r = 0; r <= g->rounds; ++r) {
        GTRY(get(&g->hv[r], nH));
        GTRY(get(&g->hc[r], mH));
        GTRY(get(&g->agv[r], nH));
        GTRY(get(&g->agc[r], mH));
    }
    GTRY(get(&g->px, n));
    GTRY(get(&g->py, m));
    GTRY(get(&g->dx, n));
    GTRY(get(&g->dy, m));
    GTRY(get(&g->tx, n));
    GTRY(get(&g->ty, m));
    GTRY(get(&g->mv, H));
    GTRY(get(&g->mcm, H));
    GTRY(get(&g->logw, 4));
    GTRY(get(&g->dhv, nH));
    GTRY(get(&g->dhc, mH));
    GTRY(get(&g->dhv2, nH));
    GTRY(get(&g->dhc2, mH));
    GTRY(get(&g->dag, std::max(nH, mH)));
    const long long blocks = (std::max(n, m) + kRows - 1) / kRows;
    GTRY(get(&g->part, blocks * (long long)H * H + blocks * H));
    void* q = nullptr;
    GCU(cudaMalloc(&q, sizeof(double) * 4096));
    g->ws.push_back(q);
    g->dpart = static_cast<double*>(q);
    q = nullptr;
    GCU(cudaMalloc(&q, sizeof(double) * kMeanBlocks * H));
    g->ws.push_back(q);
    g->mpart = static_cast<double*>(q);
    g->cap_n = n;
    g->cap_m = m;
    return MC_OK;
}


// ------------------------------------------------- instance on the device
// The same graph and features as the host build (bit for bit: the same
// float sums in the same order -- a column over its entries, a row over its
// columns in ascending order -- and the same double/float conversions).
__global__ void g_col_norms(int n, const int* __restrict__ cs, const double* __restrict__ v, float* __restrict__ cv,
                            float* __restrict__ cnorm) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int p = cs[j]; p < cs[j + 1]; ++p) {
            cv[p] = (float)v[p];
            acc += (float)fabs(v[p]);
        }
        cnorm[j] = acc;
    }
}

__global__ void g_row_norms(int m, const int* __restrict__ rs, const double* __restrict__ rvd, float* __restrict__ rv,
                            float* __restrict__ rnorm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int p = rs[i]; p < rs[i + 1]; ++p) {
            rv[p] = (float)rvd[p];
            acc += (float)fabs(rvd[p]);
        }
        rnorm[i] = acc;
    }
}

// max of non-negative floats (their bit patterns order like the values)
__global__ void g_max_nonneg(long long len, const float* __restrict__ a, unsigned* __restrict__ out) {
    unsigned best = 0u;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        best = max(best, __float_as_uint(a[i]));
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void g_var_features(int n, const double* __restrict__ obj, const double* __restrict__ lo,
                               const double* __restrict__ hi, const float* __restrict__ cnorm,
                               const unsigned* __restrict__ cmax_bits, double bs, double cs, float* __restrict__ Fv,
                               float* __restrict__ cinv) {
    const float cmax = fmaxf(1e-30f, __uint_as_float(*cmax_bits));
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double l = lo[j], h = hi[j];
        float* f = Fv + (size_t)j * FV;
        f[0] = (float)(obj[j] / cs);
        f[1] = isfinite(l) ? 1.f : 0.f;
        f[2] = isfinite(h) ? 1.f : 0.f;
        f[3] = isfinite(l) ? (float)fmax(-10.0, fmin(10.0, l / bs)) : 0.f;
        f[4] = isfinite(h) ? (float)fmax(-10.0, fmin(10.0, h / bs)) : 0.f;
        f[5] = cnorm[j] / cmax;
        cinv[j] = cnorm[j] > 0.f ? 1.f / cnorm[j] : 0.f;
    }
}

__global__ void g_row_features(int m, const double* __restrict__ lo, const double* __restrict__ hi,
                               const float* __restrict__ rnorm, const unsigned* __restrict__ rmax_bits, double bs,
                               float* __restrict__ Fc, float* __restrict__ rinv) {
    const float rmax = fmaxf(1e-30f, __uint_as_float(*rmax_bits));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const double l = lo[i], h = hi[i];
        float* f = Fc + (size_t)i * FC;
        f[0] = isfinite(l) ? (float)(l / bs) : 0.f;
        f[1] = isfinite(h) ? (float)(h / bs) : 0.f;
        f[2] = isfinite(l) ? 1.f : 0.f;
        f[3] = isfinite(h) ? 1.f : 0.f;
        f[4] = rnorm[i] / rmax;
        rinv[i] = rnorm[i] > 0.f ? 1.f / rnorm[i] : 0.f;
    }
}

__global__ void g_check_csc(int m, int n, long long nnz, const int* __restrict__ cs, const int* __restrict__ ri,
                            int* __restrict__ bad) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int b = cs[j], e = cs[j + 1];
        if ((j == 0 && b != 0) || (j == n - 1 && (long long)e != nnz) || b < 0 || b > e || (long long)e > nnz) {
            atomicOr(bad, 1);
            continue;
        }
        for (int p = b; p < e; ++p)
            if (ri[p] < 0 || ri[p] >= m) atomicOr(bad, 2);
    }
}

// Large instances (at least 2^20 nonzeros; the environment variable
// MC_GNN_DEVICE_BUILD_MIN_NNZ moves the threshold) are built on the device:
// the engine's transpose for the CSR, then norms and features in kernels.
long long device_build_min_nnz() {
    const char* e = std::getenv("MC_GNN_DEVICE_BUILD_MIN_NNZ");
    return e ? std::atoll(e) : (1LL << 20);
}

int load_instance_device(mc_gnn* g, const mc_lp* lp, Instance& I) {
    cudaStream_t s = g->stream;
    const int m = I.m, n = I.n;
    const long long nnz = I.nnz;
    if (!g->aux) {
        g->aux = mc::aux_ctx_create(g->device);
        if (!g->aux) return mc::set_error(MC_ERR_CUDA, "auxiliary context for the network's transpose");
    }
    double bs = 1.0, cs = 1.0;  // |b|_inf and |c|_inf, as the host build takes them
    for (int i = 0; i < m; ++i) {
        if (std::isfinite(lp->row_lower[i])) bs = std::max(bs, std::fabs(lp->row_lower[i]));
        if (std::isfinite(lp->row_upper[i])) bs = std::max(bs, std::fabs(lp->row_upper[i]));
    }
    for (int j = 0; j < n; ++j) cs = std::max(cs, std::fabs(lp->objective[j]));
    I.bscale = bs;
    I.cscale = cs;
    Instance T(g->device, s);  // staging, freed on return
    double *v = nullptr, *rvd = nullptr, *obj = nullptr, *vlo = nullptr, *vhi = nullptr, *rlo = nullptr,
           *rhi = nullptr;
    float *cnorm = nullptr, *rnorm = nullptr;
    unsigned* maxes = nullptr;
    int* bad = nullptr;
    GTRY(T.alloc(&v, nnz));
    GTRY(T.alloc(&rvd, nnz));
    GTRY(T.alloc(&obj, n));
    GTRY(T.alloc(&vlo, n));
    GTRY(T.alloc(&vhi, n));
    GTRY(T.alloc(&rlo, m));
    GTRY(T.alloc(&rhi, m));
    GTRY(T.alloc(&cnorm, n));
    GTRY(T.alloc(&rnorm, m));
    GTRY(T.alloc(&maxes, 2));
    GTRY(T.alloc(&bad, 1));
    GTRY(I.alloc(&I.cs, n + 1));
    GTRY(I.alloc(&I.ri, nnz));
    GTRY(I.alloc(&I.cv, nnz));
    GTRY(I.alloc(&I.rs, m + 1));
    GTRY(I.alloc(&I.ci, nnz));
    GTRY(I.alloc(&I.rv, nnz));
    GTRY(I.alloc(&I.rinv, m));
    GTRY(I.alloc(&I.cinv, n));
    GTRY(I.alloc(&I.Fv, (long long)n * FV));
    GTRY(I.alloc(&I.Fc, (long long)m * FC));
    GCU(cudaMemcpyAsync(I.cs, lp->col_start, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.ri, lp->row_index, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(v, lp->value, sizeof(double) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(obj, lp->objective, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(vlo, lp->var_lower, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(vhi, lp->var_upper, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(rlo, lp->row_lower, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(rhi, lp->row_upper, sizeof(double) * m, cudaMemcpyHostToDevice, s));
    GCU(cudaMemsetAsync(bad, 0, sizeof(int), s));
    GCU(cudaMemsetAsync(maxes, 0, sizeof(unsigned) * 2, s));
    g_check_csc<<<grid_of(n), kThreads, 0, s>>>(m, n, nnz, I.cs, I.ri, bad);
    int hb = 0;
    GCU(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    GCU(cudaStreamSynchronize(s));
    if (hb) return mc::set_error(MC_ERR_INVALID_ARGUMENT, hb & 2 ? "row index out of range" : "invalid CSC offsets");
    GTRY(mc::aux_csr(g->aux, m, n, nnz, I.cs, I.ri, v, I.rs, I.ci, rvd));
    g_col_norms<<<grid_of(n), kThreads, 0, s>>>(n, I.cs, v, I.cv, cnorm);
    g_row_norms<<<grid_of(m), kThreads, 0, s>>>(m, I.rs, rvd, I.rv, rnorm);
    g_max_nonneg<<<grid_of(n), kThreads, 0, s>>>(n, cnorm, maxes);
    g_max_nonneg<<<grid_of(m), kThreads, 0, s>>>(m, rnorm, maxes + 1);
    g_var_features<<<grid_of(n), kThreads, 0, s>>>(n, obj, vlo, vhi, cnorm, maxes, bs, cs, I.Fv, I.cinv);
    g_row_features<<<grid_of(m), kThreads, 0, s>>>(m, rlo, rhi, rnorm, maxes + 1, bs, I.Fc, I.rinv);
    GCU(cudaGetLastError());
    GCU(cudaStreamSynchronize(s));  // the staging buffers are freed on return
    return MC_OK;
}

// Graph and features of an LP given in host memory.
int load_instance(mc_gnn* g, const mc_lp* lp, Instance& I) {
    cudaStream_t s = g->stream;
    if (!lp || lp->memory != MC_MEMORY_HOST)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "the network reads LPs from host memory");
    const int m = lp->num_rows, n = lp->num_cols;
    const long long nnz = lp->nnz;
    if (m <= 0 || n <= 0) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "empty LP");
    I.m = m;
    I.n = n;
    I.nnz = nnz;
    if (nnz >= device_build_min_nnz()) return load_instance_device(g, lp, I);
    // host: CSR (stable counting sort keeps columns ascending), norms, features
    std::vector<int> rs(m + 1, 0), ci(nnz);
    std::vector<float> rv(nnz), cv(nnz), rnorm(m, 0.f), cnorm(n, 0.f);
    for (long long p = 0; p < nnz; ++p) {
        const int r = lp->row_index[p];
        if (r < 0 || r >= m) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "row index out of range");
        rs[r + 1]++;
    }
    for (int i = 0; i < m; ++i) rs[i + 1] += rs[i];
    std::vector<int> cur(rs.begin(), rs.end() - 1);
    for (int j = 0; j < n; ++j)
        for (int p = lp->col_start[j]; p < lp->col_start[j + 1]; ++p) {
            const int r = lp->row_index[p];
            const int q = cur[r]++;
            ci[q] = j;
            rv[q] = (float)lp->value[p];
            cv[p] = (float)lp->value[p];
            rnorm[r] += (float)std::fabs(lp->value[p]);
            cnorm[j] += (float)std::fabs(lp->value[p]);
        }
    double bs = 1.0, cs = 1.0;
    for (int i = 0; i < m; ++i) {
        if (std::isfinite(lp->row_lower[i])) bs = std::max(bs, std::fabs(lp->row_lower[i]));
        if (std::isfinite(lp->row_upper[i])) bs = std::max(bs, std::fabs(lp->row_upper[i]));
    }
    for (int j = 0; j < n; ++j) cs = std::max(cs, std::fabs(lp->objective[j]));
    I.bscale = bs;
    I.cscale = cs;
    float rmax = 1e-30f, cmax = 1e-30f;
    for (float v : rnorm) rmax = std::max(rmax, v);
    for (float v : cnorm) cmax = std::max(cmax, v);
    std::vector<float> Fv((size_t)n * FV), Fc((size_t)m * FC), rinv(m), cinv(n);
    for (int j = 0; j < n; ++j) {
        const double l = lp->var_lower[j], h = lp->var_upper[j];
        float* f = &Fv[(size_t)j * FV];
        f[0] = (float)(lp->objective[j] / cs);
        f[1] = std::isfinite(l) ? 1.f : 0.f;
        f[2] = std::isfinite(h) ? 1.f : 0.f;
        f[3] = std::isfinite(l) ? (float)std::max(-10.0, std::min(10.0, l / bs)) : 0.f;
        f[4] = std::isfinite(h) ? (float)std::max(-10.0, std::min(10.0, h / bs)) : 0.f;
        f[5] = cnorm[j] / cmax;
        cinv[j] = cnorm[j] > 0.f ? 1.f / cnorm[j] : 0.f;
    }
    for (int i = 0; i < m; ++i) {
        const double l = lp->row_lower[i], h = lp->row_upper[i];
        float* f = &Fc[(size_t)i * FC];
        f[0] = std::isfinite(l) ? (float)(l / bs) : 0.f;
        f[1] = std::isfinite(h) ? (float)(h / bs) : 0.f;
        f[2] = std::isfinite(l) ? 1.f : 0.f;
        f[3] = std::isfinite(h) ? 1.f : 0.f;
        f[4] = rnorm[i] / rmax;
        rinv[i] = rnorm[i] > 0.f ? 1.f / rnorm[i] : 0.f;
    }
    GTRY(I.alloc(&I.cs, n + 1));
    GTRY(I.alloc(&I.ri, nnz));
    GTRY(I.alloc(&I.cv, nnz));
    GTRY(I.alloc(&I.rs, m + 1));
    GTRY(I.alloc(&I.ci, nnz));
    GTRY(I.alloc(&I.rv, nnz));
    GTRY(I.alloc(&I.rinv, m));
    GTRY(I.alloc(&I.cinv, n));
    GTRY(I.alloc(&I.Fv, (long long)n * FV));
    GTRY(I.alloc(&I.Fc, (long long)m * FC));
    GCU(cudaMemcpyAsync(I.cs, lp->col_start, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.ri, lp->row_index, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.cv, cv.data(), sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.rs, rs.data(), sizeof(int) * (m + 1), cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.ci, ci.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.rv, rv.data(), sizeof(float) * nnz, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.rinv, rinv.data(), sizeof(float) * m, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.cinv, cinv.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.Fv, Fv.data(), sizeof(float) * Fv.size(), cudaMemcpyHostToDevice, s));
    GCU(cudaMemcpyAsync(I.Fc, Fc.data(), sizeof(float) * Fc.size(), cudaMemcpyHostToDevice, s));
    GCU(cudaStreamSynchronize(s));  // host staging vectors go out of scope
    return MC_OK;
}

int forward(mc_gnn* g, const Instance& I) {
    cudaStream_t s = g->stream;
    const float* P = g->params;
    const Layout& L = g->L;
    const int n = I.n, m = I.m;
    g_dense_fwd<<<tile_grid(n), kThreads, 0, s>>>(n, I.Fv, FV, P + L.Wve, nullptr, 0, nullptr,
                                                               P + L.bve, g->hv[0], 1);
    g_dense_fwd<<<tile_grid(m), kThreads, 0, s>>>(m, I.Fc, FC, P + L.Wce, nullptr, 0, nullptr,
                                                               P + L.bce, g->hc[0], 1);
    for (int r = 1; r <= g->rounds; ++r) {
        // constraints gather variables: agc_i = sum_j a_ij / |A_i| hv_j
        g_aggregate<<<grid_of((long long)m * 32), kThreads, 0, s>>>(m, I.rs, I.ci, I.rv, I.rinv, nullptr,
                                                                     g->hv[r - 1], g->agc[r], 0);
        g_dense_fwd<<<tile_grid(m), kThreads, 0, s>>>(m, g->hc[r - 1], H, P + L.Wcs[r - 1], g->agc[r], H,
                                                                   P + L.Wcn[r - 1], P + L.bc[r - 1], g->hc[r], 1);
        // variables gather constraints: agv_j = sum_i a_ij / |A_j| hc_i
        g_aggregate<<<grid_of((long long)n * 32), kThreads, 0, s>>>(n, I.cs, I.ri, I.cv, I.cinv, nullptr,
                                                                     g->hc[r], g->agv[r], 0);
        g_dense_fwd<<<tile_grid(n), kThreads, 0, s>>>(n, g->hv[r - 1], H, P + L.Wvs[r - 1], g->agv[r], H,
                                                                   P + L.Wvn[r - 1], P + L.bv[r - 1], g->hv[r], 1);
    }
    const int R = g->rounds;
    g_readout<<<grid_of(n), kThreads, 0, s>>>(n, g->hv[R], P + L.wx, P + L.bx, g->px);
    g_readout<<<grid_of(m), kThreads, 0, s>>>(m, g->hc[R], P + L.wy, P + L.by, g->py);
    g_col_sum_parts<<<kMeanBlocks, kThreads, 0, s>>>(n, g->hv[R], g->mpart);
    g_col_mean<<<1, H, 0, s>>>(n, kMeanBlocks, g->mpart, g->mv);
    g_col_sum_parts<<<kMeanBlocks, kThreads, 0, s>>>(m, g->hc[R], g->mpart);
    g_col_mean<<<1, H, 0, s>>>(m, kMeanBlocks, g->mpart, g->mcm);
    GCU(cudaGetLastError());
    return MC_OK;
}

// log omega on the host from the pooled means (64-long dots)
int log_omega(mc_gnn* g, double* out) {
    float mv[H], mcm[H], uv[H], uc[H], bw;
    const Layout& L = g->L;
    GCU(cudaMemcpyAsync(mv, g->mv, sizeof mv, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaMemcpyAsync(mcm, g->mcm, sizeof mcm, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaMemcpyAsync(uv, g->params + L.uv, sizeof uv, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaMemcpyAsync(uc, g->params + L.uc, sizeof uc, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaMemcpyAsync(&bw, g->params + L.bw, sizeof bw, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaStreamSynchronize(g->stream));
    double acc = bw;
    for (int c = 0; c < H; ++c) acc += (double)mv[c] * uv[c] + (double)mcm[c] * uc[c];
    *out = acc;
    return MC_OK;
}

int weight_grad(mc_gnn* g, int N, const float* X, int K, const float* dZ, long long w_off, long long b_off) {
    cudaStream_t s = g->stream;
    const int blocks = (N + kRows - 1) / kRows;
    float* pw = g->part;
    float* pb = g->part + (long long)blocks * K * H;
    g_dense_bwd_w<<<blocks, kThreads, 0, s>>>(N, X, K, dZ, pw, b_off >= 0 ? pb : nullptr);
    g_reduce_parts<<<grid_of(K * H), kThreads, 0, s>>>(blocks, K * H, pw, g->grads + w_off);
    if (b_off >= 0) g_reduce_parts<<<1, H, 0, s>>>(blocks, H, pb, g->grads + b_off);
    GCU(cudaGetLastError());
    return MC_OK;
}

// Forward, loss, backward into g->grads (zeroed first).  Targets in model units.
int loss_and_grad(mc_gnn* g, const Instance& I, double target_logw, double* loss_out) {
    cudaStream_t s = g->stream;
    const Layout& L = g->L;
    const float* P = g->params;
    const int n = I.n, m = I.m, R = g->rounds;
    GTRY(forward(g, I));
    GCU(cudaMemsetAsync(g->grads, 0, sizeof(float) * L.total, s));
    // losses and d predictions
    const int bx = std::min(grid_of(n), 2048), by = std::min(grid_of(m), 2048);
    g_mse<<<bx, kThreads, 0, s>>>(n, g->px, g->tx, g->dx, g->dpart);
    g_mse<<<by, kThreads, 0, s>>>(m, g->py, g->ty, g->dy, g->dpart + 2048);
    std::vector<double> parts(4096);
    GCU(cudaMemcpyAsync(parts.data(), g->dpart, sizeof(double) * 4096, cudaMemcpyDeviceToHost, s));
    double lw = 0.0;
    GTRY(log_omega(g, &lw));  // synchronises
    double lx = 0.0, ly = 0.0;
    for (int b = 0; b < bx; ++b) lx += parts[b];
    for (int b = 0; b < by; ++b) ly += parts[2048 + b];
    lx /= n;
    ly /= m;
    const double ew = lw - target_logw;
    *loss_out = lx + ly + 0.1 * ew * ew;
    const float dlw = (float)(0.2 * ew);
    // omega readout: d uv = dlw * mv, d uc = dlw * mc, d bw = dlw; d hv += dlw uv / n, d hc += dlw uc / m
    {
        float mv[H], mcm[H], gu[2 * H + 1];
        GCU(cudaMemcpyAsync(mv, g->mv, sizeof mv, cudaMemcpyDeviceToHost, s));
        GCU(cudaMemcpyAsync(mcm, g->mcm, sizeof mcm, cudaMemcpyDeviceToHost, s));
        GCU(cudaStreamSynchronize(s));
        for (int c = 0; c < H; ++c) {
            gu[c] = dlw * mv[c];
            gu[H + c] = dlw * mcm[c];
        }
        gu[2 * H] = dlw;
        GCU(cudaMemcpyAsync(g->grads + L.uv, gu, sizeof(float) * H, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(g->grads + L.uc, gu + H, sizeof(float) * H, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(g->grads + L.bw, gu + 2 * H, sizeof(float), cudaMemcpyHostToDevice, s));
        float su[2 * H];
        GCU(cudaMemcpyAsync(su, P + L.uv, sizeof(float) * H, cudaMemcpyDeviceToHost, s));
        GCU(cudaMemcpyAsync(su + H, P + L.uc, sizeof(float) * H, cudaMemcpyDeviceToHost, s));
        GCU(cudaStreamSynchronize(s));
        for (int c = 0; c < H; ++c) {
            su[c] = dlw * su[c] / n;
            su[H + c] = dlw * su[H + c] / m;
        }
        GCU(cudaMemcpyAsync(g->dag, su, sizeof(float) * 2 * H, cudaMemcpyHostToDevice, s));
        // d hv[R] = dx wx + dlw uv / n ; d hc[R] = dy wy + dlw uc / m
        g_outer_add<<<grid_of((long long)n * H), kThreads, 0, s>>>(n, g->dx, P + L.wx, g->dag, g->dhv, 0);
        g_outer_add<<<grid_of((long long)m * H), kThreads, 0, s>>>(m, g->dy, P + L.wy, g->dag + H, g->dhc, 0);
        GCU(cudaStreamSynchronize(s));  // g->dag is rewritten below
    }
    // readout weights: d wx = sum dx hv, d bx = sum dx
    {
        const int blocks = (n + kRows - 1) / kRows;
        g_readout_bwd<<<blocks, kThreads, 0, s>>>(n, g->hv[R], g->dx, g->part, g->part + (long long)blocks * H);
        g_reduce_parts<<<1, H, 0, s>>>(blocks, H, g->part, g->grads + L.wx);
        g_reduce_parts<<<1, 1, 0, s>>>(blocks, 1, g->part + (long long)blocks * H, g->grads + L.bx);
        const int bm = (m + kRows - 1) / kRows;
        g_readout_bwd<<<bm, kThreads, 0, s>>>(m, g->hc[R], g->dy, g->part + 2LL * blocks * H + blocks,
                                              g->part + 2LL * blocks * H + blocks + (long long)bm * H);
        g_reduce_parts<<<1, H, 0, s>>>(bm, H, g->part + 2LL * blocks * H + blocks, g->grads + L.wy);
        g_reduce_parts<<<1, 1, 0, s>>>(bm, 1, g->part + 2LL * blocks * H + blocks + (long long)bm * H,
                                       g->grads + L.by);
        GCU(cudaGetLastError());
    }
    // rounds, last to first.  dhv / dhc hold d h[r]; dhv2 / dhc2 build d h[r-1].
    for (int r = R; r >= 1; --r) {
        // variable update: hv[r] = relu(hv[r-1] Wvs + agv[r] Wvn + bv)
        g_relu_bwd<<<grid_of((long long)n * H), kThreads, 0, s>>>((long long)n * H, g->hv[r], g->dhv);
        GTRY(weight_grad(g, n, g->hv[r - 1], H, g->dhv, L.Wvs[r - 1], L.bv[r - 1]));
        GTRY(weight_grad(g, n, g->agv[r], H, g->dhv, L.Wvn[r - 1], -1));
        g_dense_bwd_x<<<tile_grid(n), kThreads, 0, s>>>(n, g->dhv, P + L.Wvs[r - 1], H, g->dhv2, 0);
        g_dense_bwd_x<<<tile_grid(n), kThreads, 0, s>>>(n, g->dhv, P + L.Wvn[r - 1], H, g->dag, 0);
        // agv[r]_j = sum_i a_ij cinv_j hc[r]_i  ->  d hc[r]_i += sum_j a_ij cinv_j d agv_j (CSR)
        g_aggregate<<<grid_of((long long)m * 32), kThreads, 0, s>>>(m, I.rs, I.ci, I.rv, nullptr, I.cinv, g->dag,
                                                                     g->dhc, 1);
        // constraint update: hc[r] = relu(hc[r-1] Wcs + agc[r] Wcn + bc)
        g_relu_bwd<<<grid_of((long long)m * H), kThreads, 0, s>>>((long long)m * H, g->hc[r], g->dhc);
        GTRY(weight_grad(g, m, g->hc[r - 1], H, g->dhc, L.Wcs[r - 1], L.bc[r - 1]));
        GTRY(weight_grad(g, m, g->agc[r], H, g->dhc, L.Wcn[r - 1], -1));
        g_dense_bwd_x<<<tile_grid(m), kThreads, 0, s>>>(m, g->dhc, P + L.Wcs[r - 1], H, g->dhc2, 0);
        g_dense_bwd_x<<<tile_grid(m), kThreads, 0, s>>>(m, g->dhc, P + L.Wcn[r - 1], H, g->dag, 0);
        // agc[r]_i = sum_j a_ij rinv_i hv[r-1]_j  ->  d hv[r-1]_j += sum_i a_ij rinv_i d agc_i (CSC)
        g_aggregate<<<grid_of((long long)n * 32), kThreads, 0, s>>>(n, I.cs, I.ri, I.cv, nullptr, I.rinv, g->dag,
                                                                     g->dhv2, 1);
        std::swap(g->dhv, g->dhv2);
        std::swap(g->dhc, g->dhc2);
    }
    // encoders
    g_relu_bwd<<<grid_of((long long)n * H), kThreads, 0, s>>>((long long)n * H, g->hv[0], g->dhv);
    GTRY(weight_grad(g, n, I.Fv, FV, g->dhv, L.Wve, L.bve));
    g_relu_bwd<<<grid_of((long long)m * H), kThreads, 0, s>>>((long long)m * H, g->hc[0], g->dhc);
    GTRY(weight_grad(g, m, I.Fc, FC, g->dhc, L.Wce, L.bce));
    GCU(cudaGetLastError());
    return MC_OK;
}

int set_targets(mc_gnn* g, const Instance& I, const double* x_target, const double* y_target) {
    std::vector<float> tx(I.n), ty(I.m);
    for (int j = 0; j < I.n; ++j) tx[j] = (float)(x_target[j] / I.bscale);
    for (int i = 0; i < I.m; ++i) ty[i] = (float)(y_target[i] / I.cscale);
    GCU(cudaMemcpyAsync(g->tx, tx.data(), sizeof(float) * I.n, cudaMemcpyHostToDevice, g->stream));
    GCU(cudaMemcpyAsync(g->ty, ty.data(), sizeof(float) * I.m, cudaMemcpyHostToDevice, g->stream));
    GCU(cudaStreamSynchronize(g->stream));
    return MC_OK;
}

struct Guard {
    int prev = -1;
    explicit Guard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(dev);
    }
    ~Guard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

int mc_gnn_create(int device, int rounds, uint64_t seed, mc_gnn** out) {
    if (!out || rounds < 1 || rounds > 8) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad GNN arguments");
    *out = nullptr;
    Guard guard(device);
    auto* g = new (std::nothrow) mc_gnn();
    if (!g) return mc::set_error(MC_ERR_OUT_OF_MEMORY, "host allocation failed");
    g->device = device;
    g->rounds = rounds;
    g->L = Layout(rounds);
    const long long P = g->L.total;
    std::vector<float> init(P, 0.f);
    // Glorot-uniform weights from splitmix64, zero biases
    uint64_t st = seed * 0x9E3779B97F4A7C15ULL + 1;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1.0p-53;
    };
    auto fill = [&](long long off, int fan_in, int fan_out) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (long long q = 0; q < (long long)fan_in * fan_out; ++q) init[off + q] = (float)((2.0 * uni() - 1.0) * a);
    };
    const Layout& L = g->L;
    fill(L.Wve, FV, H);
    fill(L.Wce, FC, H);
    for (int r = 0; r < rounds; ++r) {
        fill(L.Wcs[r], H, H);
        fill(L.Wcn[r], H, H);
        fill(L.Wvs[r], H, H);
        fill(L.Wvn[r], H, H);
    }
    fill(L.wx, H, 1);
    fill(L.wy, H, 1);
    fill(L.uv, H, 1);
    fill(L.uc, H, 1);
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    for (float** p : {&g->params, &g->grads, &g->m1, &g->m2})
        if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(p), sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMemcpy(g->params, init.data(), sizeof(float) * P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(g->m1, 0, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMemset(g->m2, 0, sizeof(float) * P);
    if (e != cudaSuccess) {
        delete g;
        return mc::set_error(e == cudaErrorMemoryAllocation ? MC_ERR_OUT_OF_MEMORY
                             : e == cudaErrorNoDevice ? MC_ERR_NO_DEVICE : MC_ERR_CUDA,
                             "mc_gnn_create: %s", cudaGetErrorString(e));
    }
    *out = g;
    return MC_OK;
}

int mc_gnn_destroy(mc_gnn* g) {
    delete g;
    return MC_OK;
}

int mc_gnn_num_params(const mc_gnn* g, int64_t* count) {
    if (!g || !count) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad arguments");
    *count = g->L.total;
    return MC_OK;
}

int mc_gnn_get_params(mc_gnn* g, float* host_out) {
    if (!g || !host_out) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad arguments");
    Guard guard(g->device);
    GCU(cudaMemcpyAsync(host_out, g->params, sizeof(float) * g->L.total, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaStreamSynchronize(g->stream));
    return MC_OK;
}

int mc_gnn_set_params(mc_gnn* g, const float* host_in) {
    if (!g || !host_in) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad arguments");
    Guard guard(g->device);
    GCU(cudaStreamSynchronize(g->stream));
    GCU(cudaMemcpyAsync(g->params, host_in, sizeof(float) * g->L.total, cudaMemcpyHostToDevice, g->stream));
    GCU(cudaStreamSynchronize(g->stream));
    return MC_OK;
}

int mc_gnn_predict(mc_gnn* g, const mc_lp* lp, double* x_out, double* y_out, double* log_omega_out) {
    if (!g) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "network is NULL");
    Guard guard(g->device);
    Instance I(g->device, g->stream);
    GTRY(load_instance(g, lp, I));
    GTRY(reserve_ws(g, I.n, I.m));
    GTRY(forward(g, I));
    std::vector<float> px(I.n), py(I.m);
    GCU(cudaMemcpyAsync(px.data(), g->px, sizeof(float) * I.n, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaMemcpyAsync(py.data(), g->py, sizeof(float) * I.m, cudaMemcpyDeviceToHost, g->stream));
    double lw = 0.0;
    GTRY(log_omega(g, &lw));
    if (x_out)
        for (int j = 0; j < I.n; ++j) x_out[j] = px[j] * I.bscale;
    if (y_out)
        for (int i = 0; i < I.m; ++i) y_out[i] = py[i] * I.cscale;
    if (log_omega_out) *log_omega_out = lw;
    return MC_OK;
}

int mc_gnn_loss_and_grad(mc_gnn* g, const mc_lp* lp, const double* x_target, const double* y_target,
                         double log_omega_target, double* loss, float* grad_out) {
    if (!g || !x_target || !y_target || !loss) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad arguments");
    Guard guard(g->device);
    Instance I(g->device, g->stream);
    GTRY(load_instance(g, lp, I));
    GTRY(reserve_ws(g, I.n, I.m));
    GTRY(set_targets(g, I, x_target, y_target));
    GTRY(loss_and_grad(g, I, log_omega_target, loss));
    // the network works on its own non-blocking stream: read after it drains
    if (grad_out)
        GCU(cudaMemcpyAsync(grad_out, g->grads, sizeof(float) * g->L.total, cudaMemcpyDeviceToHost, g->stream));
    GCU(cudaStreamSynchronize(g->stream));
    return MC_OK;
}

int mc_gnn_train_step(mc_gnn* g, const mc_lp* lp, const double* x_target, const double* y_target,
                      double log_omega_target, float learning_rate, double* loss) {
    double l = 0.0;
    GTRY(mc_gnn_loss_and_grad(g, lp, x_target, y_target, log_omega_target, &l, nullptr));
    Guard guard(g->device);
    g->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)g->step), c2 = 1.f - std::pow(b2, (float)g->step);
    g_adam<<<grid_of(g->L.total), kThreads, 0, g->stream>>>(g->L.total, g->params, g->grads, g->m1, g->m2,
                                                           learning_rate, b1, b2, 1e-8f, c1, c2);
    GCU(cudaGetLastError());
    GCU(cudaStreamSynchronize(g->stream));
    if (loss) *loss = l;
    return MC_OK;
}

}  // extern "C"
