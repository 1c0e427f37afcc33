// Binary CSC model files: the ingestion path for models beyond the reference
// MPS reader's limits (include/markov_cero/io/mps.hpp:13-20: 16 MiB, 1M rows
// and columns, 20M nonzeros).  Host code only.
//
// Layout (little-endian), a 64-byte header then the arrays back to back:
//   char  magic[8] = "MCLPCSC1"
//   int32 num_rows, int32 num_cols, int64 nnz
//   int32 objective_sense, int32 reserved (0)
//   double objective_offset
//   uint8 pad[24] (0)
//   int32 col_start[n+1], int32 row_index[nnz], double value[nnz],
//   double objective[n], var_lower[n], var_upper[n], row_lower[m], row_upper[m]
// Infinite bounds are IEEE infinities.  The reader checks the header and the
// file length; the solver validates the arrays themselves on the device.
//
// Reading into device memory streams the file through two pinned staging
// buffers (one read while the other is copied), so a model of any size loads
// with a few MiB of host memory.
#include "mc_pdlp.h"

#include <cuda_runtime.h>

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace mc {
int set_error(int code, const char* fmt, ...);
}

namespace {

constexpr char kMagic[8] = {'M', 'C', 'L', 'P', 'C', 'S', 'C', '1'};
constexpr size_t kHeader = 64;
constexpr size_t kStage = 8u << 20;  // bytes per pinned staging buffer

struct Header {
    char magic[8];
    int32_t m, n;
    int64_t nnz;
    int32_t sense, reserved;
    double offset;
    uint8_t pad[24];
};
static_assert(sizeof(Header) == kHeader, "header layout");

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

long long payload_bytes(const Header& h) {
    const long long m = h.m, n = h.n, z = h.nnz;
    return 4 * (n + 1) + 4 * z + 8 * z + 8 * 3 * n + 8 * 2 * m;
}

int read_header(File& file, const char* path, Header& h) {
    if (!path) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "model file path is NULL");
    file.f = std::fopen(path, "rb");
    if (!file.f) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "cannot open %s: %s", path, std::strerror(errno));
    if (std::fread(&h, 1, kHeader, file.f) != kHeader || std::memcmp(h.magic, kMagic, 8) != 0)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s is not an MCLPCSC1 model file", path);
    if (h.m < 0 || h.n < 0 || h.nnz < 0 || (h.sense != MC_MINIMIZE && h.sense != MC_MAXIMIZE))
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s: bad header (m %d, n %d, nnz %lld)", path, h.m, h.n,
                             (long long)h.nnz);
    if (h.nnz >= (1LL << 31) - 1) return mc::set_error(MC_ERR_RESOURCE_LIMIT, "%s: nnz beyond int32 indices", path);
    if (std::fseek(file.f, 0, SEEK_END) != 0) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s: seek failed", path);
    const long long size = std::ftell(file.f);
    if (size != (long long)kHeader + payload_bytes(h))
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s: %lld bytes, header says %lld", path, size,
                             (long long)kHeader + payload_bytes(h));
    if (std::fseek(file.f, (long)kHeader, SEEK_SET) != 0)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s: seek failed", path);
    return MC_OK;
}

// Copy `bytes` from the file into dst (host, or device through the staging pair).
struct Reader {
    File* file;
    bool device;
    void* stage[2] = {nullptr, nullptr};
    cudaStream_t stream = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    int next = 0;

    int init() {
        if (!device) return MC_OK;
        for (int q = 0; q < 2; ++q) {
            if (cudaMallocHost(&stage[q], kStage) != cudaSuccess)
                return mc::set_error(MC_ERR_OUT_OF_MEMORY, "pinned staging buffer");
            if (cudaEventCreateWithFlags(&done[q], cudaEventDisableTiming) != cudaSuccess)
                return mc::set_error(MC_ERR_CUDA, "cudaEventCreate");
        }
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
            return mc::set_error(MC_ERR_CUDA, "cudaStreamCreate");
        return MC_OK;
    }
    ~Reader() {
        if (stream) cudaStreamSynchronize(stream);
        for (int q = 0; q < 2; ++q) {
            if (done[q]) cudaEventDestroy(done[q]);
            if (stage[q]) cudaFreeHost(stage[q]);
        }
        if (stream) cudaStreamDestroy(stream);
    }
    int copy(void* dst, size_t bytes, const char* what) {
        if (bytes == 0) return MC_OK;
        if (!dst) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "destination of %s is NULL", what);
        if (!device) {
            if (std::fread(dst, 1, bytes, file->f) != bytes)
                return mc::set_error(MC_ERR_INVALID_ARGUMENT, "short read of %s", what);
            return MC_OK;
        }
        char* out = static_cast<char*>(dst);
        for (size_t at = 0; at < bytes;) {
            const size_t chunk = bytes - at < kStage ? bytes - at : kStage;
            const int q = next;
            next ^= 1;
            // the buffer's previous copy must be done before it is refilled
            if (cudaEventSynchronize(done[q]) != cudaSuccess) return mc::set_error(MC_ERR_CUDA, "staging wait");
            if (std::fread(stage[q], 1, chunk, file->f) != chunk)
                return mc::set_error(MC_ERR_INVALID_ARGUMENT, "short read of %s", what);
            if (cudaMemcpyAsync(out + at, stage[q], chunk, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
                cudaEventRecord(done[q], stream) != cudaSuccess)
                return mc::set_error(MC_ERR_CUDA, "copy of %s to the device", what);
            at += chunk;
        }
        return MC_OK;
    }
    int finish() {
        if (device && cudaStreamSynchronize(stream) != cudaSuccess)
            return mc::set_error(MC_ERR_CUDA, "model upload");
        return MC_OK;
    }
};

int write_all(FILE* f, const void* p, size_t bytes) {
    if (bytes && (!p || std::fwrite(p, 1, bytes, f) != bytes)) return 1;
    return 0;
}

}  // namespace

extern "C" {

int mc_lp_file_write(const char* path, const mc_lp* lp) {
    if (!path || !lp) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "bad model file arguments");
    if (lp->memory != MC_MEMORY_HOST) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "the writer takes host arrays");
    if (lp->num_rows < 0 || lp->num_cols < 0 || lp->nnz < 0)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "negative model sizes");
    Header h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kMagic, 8);
    h.m = lp->num_rows;
    h.n = lp->num_cols;
    h.nnz = lp->nnz;
    h.sense = lp->objective_sense;
    h.offset = lp->objective_offset;
    File file;
    file.f = std::fopen(path, "wb");
    if (!file.f) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "cannot create %s: %s", path, std::strerror(errno));
    const size_t m = (size_t)h.m, n = (size_t)h.n, z = (size_t)h.nnz;
    int bad = write_all(file.f, &h, kHeader);
    bad |= write_all(file.f, lp->col_start, 4 * (n + 1));
    bad |= write_all(file.f, lp->row_index, 4 * z);
    bad |= write_all(file.f, lp->value, 8 * z);
    bad |= write_all(file.f, lp->objective, 8 * n);
    bad |= write_all(file.f, lp->var_lower, 8 * n);
    bad |= write_all(file.f, lp->var_upper, 8 * n);
    bad |= write_all(file.f, lp->row_lower, 8 * m);
    bad |= write_all(file.f, lp->row_upper, 8 * m);
    if (bad) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "write of %s failed", path);
    if (std::fclose(file.f) != 0) {
        file.f = nullptr;
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "close of %s failed", path);
    }
    file.f = nullptr;
    return MC_OK;
}

int mc_lp_file_info(const char* path, int32_t* num_rows, int32_t* num_cols, int64_t* nnz) {
    File file;
    Header h;
    const int rc = read_header(file, path, h);
    if (rc != MC_OK) return rc;
    if (num_rows) *num_rows = h.m;
    if (num_cols) *num_cols = h.n;
    if (nnz) *nnz = h.nnz;
    return MC_OK;
}

int mc_lp_file_read(const char* path, mc_lp* lp) {
    if (!lp) return mc::set_error(MC_ERR_INVALID_ARGUMENT, "lp is NULL");
    File file;
    Header h;
    int rc = read_header(file, path, h);
    if (rc != MC_OK) return rc;
    if (lp->num_rows != h.m || lp->num_cols != h.n || lp->nnz != h.nnz)
        return mc::set_error(MC_ERR_INVALID_ARGUMENT, "%s holds m %d n %d nnz %lld; the buffers are sized for "
                             "m %d n %d nnz %lld", path, h.m, h.n, (long long)h.nnz, lp->num_rows, lp->num_cols,
                             (long long)lp->nnz);
    Reader r{&file, lp->memory == MC_MEMORY_DEVICE};
    if ((rc = r.init()) != MC_OK) return rc;
    const size_t m = (size_t)h.m, n = (size_t)h.n, z = (size_t)h.nnz;
    // the mc_lp arrays are const for the solver; the reader fills them
    if ((rc = r.copy(const_cast<int32_t*>(lp->col_start), 4 * (n + 1), "col_start")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<int32_t*>(lp->row_index), 4 * z, "row_index")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->value), 8 * z, "value")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->objective), 8 * n, "objective")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->var_lower), 8 * n, "var_lower")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->var_upper), 8 * n, "var_upper")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->row_lower), 8 * m, "row_lower")) != MC_OK) return rc;
    if ((rc = r.copy(const_cast<double*>(lp->row_upper), 8 * m, "row_upper")) != MC_OK) return rc;
    if ((rc = r.finish()) != MC_OK) return rc;
    lp->objective_offset = h.offset;
    lp->objective_sense = h.sense;
    return MC_OK;
}

}  // extern "C"
