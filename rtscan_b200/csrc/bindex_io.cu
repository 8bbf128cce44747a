// BinDex on disk: save a column's index and load it back without the sort.
//
// The reference rebuilds every index at start-up (init_bindex_in_GPU per
// column in its driver, bindex_cuda.cpp:1769-1781): a radix sort of the
// column and K-1 filter-vector passes.  A served table that restarts can
// instead stream the index from a file at disk/PCIe speed.
//
// File layout (little-endian):
//   header   magic "RTSBDX1\0", u32 version (1), u32 K, u64 n,
//            u64 fv_stride (words per filter vector), u64 nsample,
//            u32 min_val, u32 max_val, u64 payload_bytes,
//            u64 checksum[6] of the six arrays below, u64 header_check
//   payload  u32 start[K], u64 first_rank[K], u32 sample[nsample],
//            u32 sval[n], u32 spos[n], u32 fv[(K-1) * fv_stride]
// Each checksum is sum_i mix(i, word_i) mod 2^64 over the array's 32-bit
// words (order-dependent, computed on the device for the large arrays);
// header_check is the same function over the header's preceding words.
// Loading verifies every checksum, then checks the whole index against the
// resident column on the device, so that a file whose checksums agree but
// whose contents are wrong (written by a faulty build, or crafted) is
// refused rather than answering queries wrongly or sending the refine past
// the sorted arrays: col[spos[r]] == sval[r] and sval is non-decreasing for
// every rank r; start[k] == sval[k * (n / K)]; first_rank[k] is the lower
// bound of start[k] in sval; sample[j] == sval[j * 1024]; min/max are the
// first and last sorted values; every filter-vector word equals the one
// the start values give for the column, and the padding words are zero.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rts_internal.h"

namespace rts {
namespace {

constexpr char kMagic[8] = {'R', 'T', 'S', 'B', 'D', 'X', '1', '\0'};
constexpr uint32_t kVersion = 1;

struct FileHeader {
  char magic[8];
  uint32_t version;
  uint32_t K;
  uint64_t n;
  uint64_t fv_stride;
  uint64_t nsample;
  uint32_t min_val;
  uint32_t max_val;
  uint64_t payload_bytes;
  uint64_t checksum[6];  // start, first_rank, sample, sval, spos, fv
  uint64_t header_check;
};
static_assert(sizeof(FileHeader) == 8 + 4 + 4 + 8 * 3 + 4 + 4 + 8 + 48 + 8, "packed header");

__host__ __device__ __forceinline__ uint64_t mix(uint64_t i, uint32_t w) {
  uint64_t z = (uint64_t)w + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t host_checksum(const void *p, size_t bytes) {
  const uint32_t *w = static_cast<const uint32_t *>(p);
  uint64_t s = 0;
  for (size_t i = 0; i < bytes / 4; i++) s += mix(i, w[i]);
  return s;
}

__global__ void checksum_kernel(const uint32_t *__restrict__ p, uint64_t n, unsigned long long *out) {
  uint64_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    s += mix(i, p[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)s);
}

// Counts ranks whose (value, row) pair disagrees with the column or whose
// value is below its predecessor's.
__global__ void verify_kernel(const uint32_t *__restrict__ col, const uint32_t *__restrict__ sval,
                              const uint32_t *__restrict__ spos, uint64_t n, unsigned long long *bad) {
  unsigned long long b = 0;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = sval[r], row = spos[r];
    b += row >= n || col[row] != v || (r > 0 && sval[r - 1] > v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(bad, b);
}

// Counts entries of the area table, the planner's sample and the
// filter-vector padding that disagree with the sorted values: start[k] must
// be sval[k*(n/K)], first_rank[k] its lower bound (sval[r] == start[k] and
// r == 0 or sval[r-1] < start[k]), sample[j] sval[j*stride], and every
// padding word past `words` in a filter vector zero.
__global__ void tables_kernel(const uint32_t *__restrict__ sval, uint64_t n, int K, const uint32_t *__restrict__ start,
                              const uint64_t *__restrict__ first_rank, const uint32_t *__restrict__ sample, uint64_t m,
                              uint64_t stride, const uint32_t *__restrict__ fv, uint64_t fv_stride, uint64_t words,
                              unsigned long long *bad) {
  const uint64_t pad = fv_stride - words;
  const uint64_t total = (uint64_t)K + m + (uint64_t)(K - 1) * pad;
  const uint64_t avg = n / (uint64_t)K;
  unsigned long long b = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    if (i < (uint64_t)K) {
      const uint32_t v = sval[i * avg];
      const uint64_t r = first_rank[i];
      b += start[i] != v || r > i * avg || sval[r] != v || (r > 0 && sval[r - 1] >= v);
    } else if (i < (uint64_t)K + m) {
      const uint64_t j = i - K;
      b += sample[j] != sval[j * stride];
    } else {
      const uint64_t q = i - K - m;
      b += fv[(q / pad) * fv_stride + words + q % pad] != 0;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(bad, b);
}

uint64_t device_checksum(const uint32_t *p, uint64_t words, unsigned long long *scratch, int sm_count) {
  RTS_CUDA(cudaMemset(scratch, 0, 8));
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((words + 255) / 256, (uint64_t)sm_count * 8));
  checksum_kernel<<<grid, 256>>>(p, words, scratch);
  RTS_CUDA(cudaGetLastError());
  unsigned long long v = 0;
  RTS_CUDA(cudaMemcpy(&v, scratch, 8, cudaMemcpyDeviceToHost));
  return v;
}

uint64_t header_checksum(const FileHeader &h) { return host_checksum(&h, offsetof(FileHeader, header_check)); }

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

struct Pinned {
  void *p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

constexpr size_t kStage = 16u << 20;  // bytes per staging copy

void write_all(FILE *f, const void *p, size_t bytes, const std::string &path) {
  if (bytes && fwrite(p, 1, bytes, f) != bytes) throw Error(RTS_ERR_IO, path + ": write failed");
}

void read_all(FILE *f, void *p, size_t bytes, const std::string &path) {
  if (bytes && fread(p, 1, bytes, f) != bytes) throw Error(RTS_ERR_PARSE, path + ": file is truncated");
}

void write_device(FILE *f, const uint32_t *dev, uint64_t words, void *stage, const std::string &path) {
  for (uint64_t off = 0; off < words; off += kStage / 4) {
    const size_t m = (size_t)std::min<uint64_t>(kStage / 4, words - off);
    RTS_CUDA(cudaMemcpy(stage, dev + off, m * 4, cudaMemcpyDeviceToHost));
    write_all(f, stage, m * 4, path);
  }
}

void read_device(FILE *f, uint32_t *dev, uint64_t words, void *stage, const std::string &path) {
  for (uint64_t off = 0; off < words; off += kStage / 4) {
    const size_t m = (size_t)std::min<uint64_t>(kStage / 4, words - off);
    read_all(f, stage, m * 4, path);
    RTS_CUDA(cudaMemcpy(dev + off, stage, m * 4, cudaMemcpyHostToDevice));
  }
}

FileHeader read_header(FILE *f, const std::string &path) {
  FileHeader h;
  read_all(f, &h, sizeof h, path);
  if (memcmp(h.magic, kMagic, sizeof kMagic) != 0) throw Error(RTS_ERR_PARSE, path + ": not a BinDex file");
  if (h.version != kVersion) throw Error(RTS_ERR_PARSE, path + ": unsupported BinDex file version");
  if (header_checksum(h) != h.header_check) throw Error(RTS_ERR_PARSE, path + ": header checksum mismatch");
  const uint64_t want = (uint64_t)h.K * 12 + h.nsample * 4 + h.n * 8 + (uint64_t)(h.K - 1) * h.fv_stride * 4;
  if (h.K < 2 || h.K > 4096 || h.n < h.K || h.fv_stride < ((h.n + 31) >> 5) || h.payload_bytes != want)
    throw Error(RTS_ERR_PARSE, path + ": inconsistent BinDex header");
  return h;
}

rts_status fail(rts_ctx *ctx, rts_status code, const char *what) {
  if (ctx) ctx->err = what;
  return set_thread_error(code, what);
}

}  // namespace
}  // namespace rts

extern "C" {

rts_status rts_save_bindex(rts_ctx *ctx, int32_t column, const char *path) {
  rts::Range nvtx_range_("rts_save_bindex");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!path) throw rts::Error(RTS_ERR_ARG, "null path");
    if (column < 0 || column >= (int)ctx->bindex.size() || !ctx->bindex[column])
      throw rts::Error(RTS_ERR_STATE, "column has no BinDex");
    const rts::GpuBinDex &B = *ctx->bindex[column];
    rts::DeviceGuard device_guard(ctx->device);
    unsigned long long *scratch = rts::small_device_buffer(ctx);
    rts::FileHeader h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, rts::kMagic, sizeof rts::kMagic);
    h.version = rts::kVersion;
    h.K = (uint32_t)B.K;
    h.n = B.n;
    h.fv_stride = B.fv_stride;
    h.nsample = B.sample.size();
    h.min_val = B.min_val;
    h.max_val = B.max_val;
    std::vector<uint64_t> ranks(B.first_rank.begin(), B.first_rank.end());
    h.payload_bytes = (uint64_t)B.K * 12 + h.nsample * 4 + B.n * 8 + (uint64_t)(B.K - 1) * B.fv_stride * 4;
    h.checksum[0] = rts::host_checksum(B.start.data(), B.start.size() * 4);
    h.checksum[1] = rts::host_checksum(ranks.data(), ranks.size() * 8);
    h.checksum[2] = rts::host_checksum(B.sample.data(), B.sample.size() * 4);
    h.checksum[3] = rts::device_checksum(B.sval, B.n, scratch, ctx->sm_count);
    h.checksum[4] = rts::device_checksum(B.spos, B.n, scratch, ctx->sm_count);
    h.checksum[5] = rts::device_checksum(B.fv, (uint64_t)(B.K - 1) * B.fv_stride, scratch, ctx->sm_count);
    h.header_check = rts::header_checksum(h);
    rts::File f;
    const std::string p(path);
    f.f = fopen(path, "wb");
    if (!f.f) throw rts::Error(RTS_ERR_IO, p + ": cannot create");
    rts::Pinned stage;
    RTS_CUDA(cudaMallocHost(&stage.p, rts::kStage));
    rts::write_all(f.f, &h, sizeof h, p);
    rts::write_all(f.f, B.start.data(), B.start.size() * 4, p);
    rts::write_all(f.f, ranks.data(), ranks.size() * 8, p);
    rts::write_all(f.f, B.sample.data(), B.sample.size() * 4, p);
    rts::write_device(f.f, B.sval, B.n, stage.p, p);
    rts::write_device(f.f, B.spos, B.n, stage.p, p);
    rts::write_device(f.f, B.fv, (uint64_t)(B.K - 1) * B.fv_stride, stage.p, p);
    if (fflush(f.f) != 0) throw rts::Error(RTS_ERR_IO, p + ": write failed");
    return RTS_OK;
  } catch (const rts::Error &e) {
    return rts::fail(ctx, e.code, e.what());
  } catch (const std::exception &e) {
    return rts::fail(ctx, RTS_ERR_NOMEM, e.what());
  }
}

rts_status rts_bindex_file_info(const char *path, int32_t *K, uint64_t *nrows) {
  try {
    if (!path) throw rts::Error(RTS_ERR_ARG, "null path");
    rts::File f;
    f.f = fopen(path, "rb");
    if (!f.f) throw rts::Error(RTS_ERR_IO, std::string(path) + ": cannot open");
    const rts::FileHeader h = rts::read_header(f.f, path);
    if (K) *K = (int32_t)h.K;
    if (nrows) *nrows = h.n;
    return RTS_OK;
  } catch (const std::exception &e) {
    return rts::set_thread_error(rts::status_of(e), e.what());
  }
}

rts_status rts_load_bindex(rts_ctx *ctx, int32_t column, const char *path) {
  rts::Range nvtx_range_("rts_load_bindex");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!path) throw rts::Error(RTS_ERR_ARG, "null path");
    if (ctx->cols.empty()) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (column < 0 || column >= (int)ctx->cols.size()) throw rts::Error(RTS_ERR_ARG, "column out of range");
    const std::string p(path);
    rts::File f;
    f.f = fopen(path, "rb");
    if (!f.f) throw rts::Error(RTS_ERR_IO, p + ": cannot open");
    const rts::FileHeader h = rts::read_header(f.f, p);
    if (h.n != ctx->nrows)
      throw rts::Error(RTS_ERR_PARSE, p + ": index of " + std::to_string(h.n) + " rows, table has " +
                                          std::to_string(ctx->nrows));
    if (h.fv_stride != (((h.n + 31) >> 5) + 3) / 4 * 4) throw rts::Error(RTS_ERR_PARSE, p + ": bad fv_stride");
    if (h.nsample != (h.n + rts::kSampleStride - 1) / rts::kSampleStride)
      throw rts::Error(RTS_ERR_PARSE, p + ": bad sample count");
    rts::DeviceGuard device_guard(ctx->device);
    auto b = std::make_unique<rts::GpuBinDex>();
    b->K = (int)h.K;
    b->n = h.n;
    b->fv_stride = h.fv_stride;
    b->min_val = h.min_val;
    b->max_val = h.max_val;
    b->start.resize(h.K);
    std::vector<uint64_t> ranks(h.K);
    b->sample.resize(h.nsample);
    rts::read_all(f.f, b->start.data(), h.K * 4, p);
    rts::read_all(f.f, ranks.data(), h.K * 8, p);
    rts::read_all(f.f, b->sample.data(), h.nsample * 4, p);
    if (rts::host_checksum(b->start.data(), h.K * 4) != h.checksum[0] ||
        rts::host_checksum(ranks.data(), h.K * 8) != h.checksum[1] ||
        rts::host_checksum(b->sample.data(), h.nsample * 4) != h.checksum[2])
      throw rts::Error(RTS_ERR_PARSE, p + ": checksum mismatch (area table)");
    b->first_rank.assign(ranks.begin(), ranks.end());
    auto alloc = [&](uint32_t *&dst, uint64_t words) {
      if (cudaMalloc(&dst, std::max<uint64_t>(words, 1) * 4) != cudaSuccess) {
        cudaGetLastError();
        throw rts::Error(RTS_ERR_NOMEM, "device allocation failed");
      }
    };
    alloc(b->sval, h.n);
    alloc(b->spos, h.n);
    alloc(b->fv, (uint64_t)(h.K - 1) * h.fv_stride);
    rts::Pinned stage;
    RTS_CUDA(cudaMallocHost(&stage.p, rts::kStage));
    rts::read_device(f.f, b->sval, h.n, stage.p, p);
    rts::read_device(f.f, b->spos, h.n, stage.p, p);
    rts::read_device(f.f, b->fv, (uint64_t)(h.K - 1) * h.fv_stride, stage.p, p);
    unsigned long long *scratch = rts::small_device_buffer(ctx);
    if (rts::device_checksum(b->sval, h.n, scratch, ctx->sm_count) != h.checksum[3] ||
        rts::device_checksum(b->spos, h.n, scratch, ctx->sm_count) != h.checksum[4] ||
        rts::device_checksum(b->fv, (uint64_t)(h.K - 1) * h.fv_stride, scratch, ctx->sm_count) != h.checksum[5])
      throw rts::Error(RTS_ERR_PARSE, p + ": checksum mismatch (index arrays)");
    RTS_CUDA(cudaMemset(scratch, 0, 8));
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((h.n + 255) / 256, (uint64_t)ctx->sm_count * 8));
    rts::verify_kernel<<<grid, 256>>>(ctx->cols[column], b->sval, b->spos, h.n, scratch);
    RTS_CUDA(cudaGetLastError());
    unsigned long long bad = 0;
    RTS_CUDA(cudaMemcpy(&bad, scratch, 8, cudaMemcpyDeviceToHost));
    if (bad) throw rts::Error(RTS_ERR_PARSE, p + ": index does not match column " + std::to_string(column));
    // the host tables and the filter vectors against the sorted values
    uint32_t ends[2];
    RTS_CUDA(cudaMemcpy(&ends[0], b->sval, 4, cudaMemcpyDeviceToHost));
    RTS_CUDA(cudaMemcpy(&ends[1], b->sval + h.n - 1, 4, cudaMemcpyDeviceToHost));
    if (ends[0] != h.min_val || ends[1] != h.max_val)
      throw rts::Error(RTS_ERR_PARSE, p + ": min/max do not match the sorted values");
    uint32_t *tables = nullptr;
    alloc(tables, (uint64_t)h.K * 3 + 1 + h.nsample);  // start, pad word, first_rank, sample
    struct Free {
      void *q;
      ~Free() { cudaFree(q); }
    } free_tables{tables};
    uint32_t *d_start = tables;
    uint64_t *d_rank = reinterpret_cast<uint64_t *>(tables + ((h.K + 1) & ~1u));
    uint32_t *d_sample = reinterpret_cast<uint32_t *>(d_rank + h.K);
    RTS_CUDA(cudaMemcpy(d_start, b->start.data(), h.K * 4, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemcpy(d_rank, ranks.data(), h.K * 8, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemcpy(d_sample, b->sample.data(), h.nsample * 4, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemset(scratch, 0, 8));
    const uint64_t words = (h.n + 31) >> 5;
    const uint64_t items = h.K + h.nsample + (uint64_t)(h.K - 1) * (h.fv_stride - words);
    const int tgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>((items + 255) / 256, (uint64_t)ctx->sm_count * 8));
    rts::tables_kernel<<<tgrid, 256>>>(b->sval, h.n, (int)h.K, d_start, d_rank, d_sample, h.nsample,
                                       rts::kSampleStride, b->fv, h.fv_stride, words, scratch);
    RTS_CUDA(cudaGetLastError());
    RTS_CUDA(cudaMemcpy(&bad, scratch, 8, cudaMemcpyDeviceToHost));
    if (bad) throw rts::Error(RTS_ERR_PARSE, p + ": area table or sample does not match the sorted values");
    if (rts::count_fv_mismatches(ctx->cols[column], h.n, d_start, (int)h.K, b->fv, h.fv_stride, scratch,
                                 ctx->sm_count, 0))
      throw rts::Error(RTS_ERR_PARSE, p + ": filter vectors do not match column " + std::to_string(column));
    if (ctx->bindex.size() < ctx->cols.size()) ctx->bindex.resize(ctx->cols.size());
    ctx->bindex[column] = std::move(b);
    ctx->launches += 6;  // three checksums, the order check, the tables, the filter vectors
    return RTS_OK;
  } catch (const rts::Error &e) {
    return rts::fail(ctx, e.code, e.what());
  } catch (const std::exception &e) {
    return rts::fail(ctx, RTS_ERR_NOMEM, e.what());
  }
}

}  // extern "C"
