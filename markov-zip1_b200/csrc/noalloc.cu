// Ruiz equilibration with no device allocation: mc_ruiz_equilibrate_noalloc.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// entirely owned by another allocator (a framework's caching pool, a fixed
// arena sized at start-up), where a stray cudaMalloc can fail or fragment the
// pool, or a service that must not allocate on its request path, because an
// allocation can wait on the device and its latency has no bound.  This entry point does the same
// work as mc_ruiz_equilibrate, with the same arithmetic and bit-identical
// results, but every byte of working memory it needs beyond the caller's
// inputs and outputs lives in one file-scope device array, g_ruiz_scratch,
// reserved when the library is loaded and held on every GPU that loads it
// until the process exits.
//
// Limits and behaviour:
//   * m + n <= kNoAllocMaxLines (1,048,576 rows plus columns); larger models
//     are rejected with MC_ERR_RESOURCE_LIMIT before any GPU work.  The array
//     is kNoAllocScratchBytes (about 8 MiB) per device.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (host code cannot use the array's name as a device
//     pointer) and caches it per device; make that first call before any
//     stream capture begins.  A cudaDeviceReset ends the context the cached
//     address belongs to, so the entry point must not be called on that
//     device afterwards.
//   * Without iterations_executed the call is asynchronous on its stream and
//     does not see errors raised while its kernels run.
//   * All calls share the one array: calls that may overlap on the GPU (on
//     different streams, or from different host threads) race on it and must
//     be serialised by the caller.  Each call re-initialises the parts that
//     must start from zero, so a call never sees the previous call's state.
#include "mc_pdlp.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

namespace mc {
int set_error(int code, const char* fmt, ...);
}

namespace {

constexpr int kNaBlock = 256;
constexpr int kNoAllocMaxLines = 1 << 20;  // m + n
constexpr int kNaMaxBlocks = 2048;         // grid cap of every kernel below
// layout (doubles): delta_r[m] delta_c[n] | row_err[kNaMaxBlocks] | col_err[kNaMaxBlocks] | state[8]
constexpr int kNaErrOffset = kNoAllocMaxLines;
constexpr int kNaStateOffset = kNoAllocMaxLines + 2 * kNaMaxBlocks;
constexpr int kNoAllocScratchDoubles = kNaStateOffset + 8;
constexpr size_t kNoAllocScratchBytes = sizeof(double) * kNoAllocScratchDoubles;

static __device__ __align__(256) double g_ruiz_scratch[kNoAllocScratchDoubles];

// State words inside the scratch (as long long): [0] passes, [1] converged.
struct NaState {
    long long passes;
    long long done;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device (set up once per device).
int scratch_address(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mc::set_error(MC_ERR_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return mc::set_error(MC_ERR_NO_DEVICE, "device ordinal %d beyond %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_ruiz_scratch);
        if (e != cudaSuccess || !p)
            return mc::set_error(e == cudaErrorNoKernelImageForDevice ? MC_ERR_NO_DEVICE : MC_ERR_CUDA,
                                 "cudaGetSymbolAddress(g_ruiz_scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return MC_OK;
}

__device__ __forceinline__ double na_max(double a, double b) { return (a < b) ? b : a; }

__global__ void na_init(int m, int n, double* row_scale, double* col_scale, NaState* st) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->passes = 0;
        st->done = 0;
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m + n; t += gridDim.x * blockDim.x) {
        if (t < m) row_scale[t] = 1.0;
        else col_scale[t - m] = 1.0;
    }
}

// max |a| of each line (0 -> 1) into norm[], block maxima of |1 - norm| into err[]
__global__ void na_line_max(int lines, const int* __restrict__ start, const double* __restrict__ value,
                            double* __restrict__ norm, double* __restrict__ err, const NaState* st) {
    __shared__ double red[kNaBlock / 32];
    if (st->done) return;
    double e = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        double mx = 0.0;
        for (int p = start[j]; p < start[j + 1]; ++p) mx = na_max(mx, fabs(value[p]));
        if (mx == 0.0) mx = 1.0;
        norm[j] = mx;
        e = na_max(e, fabs(1.0 - mx));
    }
    for (int off = 16; off > 0; off >>= 1) e = na_max(e, __shfl_xor_sync(0xffffffffu, e, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = na_max(b, red[w]);
        err[blockIdx.x] = b;
    }
}

// convergence test of the pass (both maxima below tolerance -> done)
__global__ void na_check(const double* __restrict__ row_err, int nrow, const double* __restrict__ col_err, int ncol,
                         double tolerance, NaState* st) {
    if (st->done || threadIdx.x != 0) return;
    double r = 0.0, c = 0.0;
    for (int b = 0; b < nrow; ++b) r = na_max(r, row_err[b]);
    for (int b = 0; b < ncol; ++b) c = na_max(c, col_err[b]);
    if (r < tolerance && c < tolerance) st->done = 1;
    else st->passes += 1;
}

// delta = 1/sqrt(norm) in place, scale *= delta
__global__ void na_deltas(int lines, double* __restrict__ norm, double* __restrict__ scale, const NaState* st) {
    if (st->done) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        const double d = 1.0 / sqrt(norm[j]);
        norm[j] = d;
        scale[j] *= d;
    }
}

// value[p] *= delta_r[row] * delta_c[col] (product formed first)
__global__ void na_rescale(int lines, const int* __restrict__ start, const int* __restrict__ inner,
                           double* __restrict__ value, const double* __restrict__ delta_outer,
                           const double* __restrict__ delta_inner, const NaState* st) {
    if (st->done) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < lines; j += gridDim.x * blockDim.x) {
        const double dout = delta_outer[j];
        for (int p = start[j]; p < start[j + 1]; ++p)
            value[p] = __dmul_rn(value[p], __dmul_rn(delta_inner[inner[p]], dout));
    }
}

__global__ void na_apply(int m, int n, const double* __restrict__ row_scale, const double* __restrict__ col_scale,
                         double* objective, double* var_lower, double* var_upper, double* row_lower,
                         double* row_upper) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
        if (t < n) {
            const double s = col_scale[t];
            const double inv = 1.0 / s;
            if (isfinite(var_lower[t])) var_lower[t] = __dmul_rn(var_lower[t], inv);
            if (isfinite(var_upper[t])) var_upper[t] = __dmul_rn(var_upper[t], inv);
            objective[t] = __dmul_rn(objective[t], s);
        } else {
            const int i = t - n;
            const double s = row_scale[i];
            if (isfinite(row_lower[i])) row_lower[i] = __dmul_rn(row_lower[i], s);
            if (isfinite(row_upper[i])) row_upper[i] = __dmul_rn(row_upper[i], s);
        }
    }
}

int grid(long long lines) {
    long long b = (lines + kNaBlock - 1) / kNaBlock;
    if (b > kNaMaxBlocks) b = kNaMaxBlocks;
    return b < 1 ? 1 : (int)b;
}

int launch_error(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return MC_OK;
    return mc::set_error(MC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace

extern "C" int mc_ruiz_equilibrate_noalloc(int32_t m, int32_t n, int64_t nnz, const int32_t* col_start,
                                           const int32_t* row_index, double* csc_value, const int32_t* row_start,
                                           const int32_t* col_index, double* csr_value, double* objective,
                                           double* var_lower, double* var_upper, double* row_lower,
                                           double* row_upper, int64_t max_iterations, double* row_scale,
                                           double* col_scale, int64_t* iterations_executed, void* stream) {
    if (m < 0 || n < 0 || nnz < 0 || max_iterations < 0 || !row_scale || !col_scale)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "mc_ruiz_equilibrate_noalloc: bad arguments");
    if ((long long)m + n > kNoAllocMaxLines)
        return mc::set_error(MC_ERR_RESOURCE_LIMIT,
                             "mc_ruiz_equilibrate_noalloc: m + n = %lld exceeds the static scratch limit of %d "
                             "rows plus columns (%zu bytes per device); use mc_ruiz_equilibrate",
                             (long long)m + n, kNoAllocMaxLines, kNoAllocScratchBytes);
    if (nnz > 0 && (!col_start || !row_index || !csc_value || !row_start || !col_index || !csr_value))
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "mc_ruiz_equilibrate_noalloc: NULL matrix array");
    double* scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != MC_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* delta_r = scratch;
    double* delta_c = scratch + m;
    double* row_err = scratch + kNaErrOffset;
    double* col_err = scratch + kNaErrOffset + kNaMaxBlocks;
    NaState* st = reinterpret_cast<NaState*>(scratch + kNaStateOffset);

    na_init<<<grid((long long)m + n), kNaBlock, 0, s>>>(m, n, row_scale, col_scale, st);
    if (m > 0 && n > 0 && nnz > 0) {
        const int gc = grid(n), gr = grid(m);
        for (long long pass = 0; pass < max_iterations; ++pass) {
            na_line_max<<<gc, kNaBlock, 0, s>>>(n, col_start, csc_value, delta_c, col_err, st);
            na_line_max<<<gr, kNaBlock, 0, s>>>(m, row_start, csr_value, delta_r, row_err, st);
            na_check<<<1, 32, 0, s>>>(row_err, gr, col_err, gc, 1e-3, st);
            na_deltas<<<gr, kNaBlock, 0, s>>>(m, delta_r, row_scale, st);
            na_deltas<<<gc, kNaBlock, 0, s>>>(n, delta_c, col_scale, st);
            na_rescale<<<gc, kNaBlock, 0, s>>>(n, col_start, row_index, csc_value, delta_c, delta_r, st);
            na_rescale<<<gr, kNaBlock, 0, s>>>(m, row_start, col_index, csr_value, delta_r, delta_c, st);
        }
        if (objective && var_lower && var_upper && row_lower && row_upper)
            na_apply<<<grid((long long)m + n), kNaBlock, 0, s>>>(m, n, row_scale, col_scale, objective, var_lower,
                                                               var_upper, row_lower, row_upper);
    }
    int lrc = launch_error("mc_ruiz_equilibrate_noalloc launch");
    if (lrc != MC_OK) return lrc;
    if (iterations_executed) {
        long long passes = 0;
        cudaError_t e = cudaMemcpyAsync(&passes, &st->passes, sizeof passes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return mc::set_error(MC_ERR_CUDA, "mc_ruiz_equilibrate_noalloc: %s", cudaGetErrorString(e));
        *iterations_executed = passes;
    }
    return MC_OK;
}
