// Internal declarations shared by the host code and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <atomic>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rtscan_b200.h"

namespace rts {

// Rows covered by one warp-tile of the fused scan: 32 lanes x 8 vectors x
// 4 values; its result is 32 bitmap words (one 128-byte store per warp).
constexpr int kTileRows = 1024;
constexpr int kTileWords = kTileRows / 32;
// Terms one fused launch evaluates; longer queries take extra AND passes.
constexpr int kFusedMaxTerms = 16;

struct Error : std::runtime_error {
  rts_status code;
  Error(rts_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define RTS_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::rts::Error(RTS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// NVTX range for the lifetime of the object: library calls and server steps
// show up by name in nsys/ncu timelines (no cost without an attached tool).
struct Range {
  explicit Range(const char *name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range &) = delete;
  Range &operator=(const Range &) = delete;
};

// Raise `kernel`'s dynamic shared-memory limit to `bytes` on the current
// device.  The attribute belongs to each device's context, so it is set once
// per device (bit d of `done`), and calls from several threads at once only
// set it twice.
template <class K>
void raise_smem_limit(K kernel, std::atomic<uint64_t> &done, int bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  RTS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.fetch_or(bit, std::memory_order_acq_rel);
}

// Make device `d` current for a scope and restore the caller's device when
// the scope ends, on error paths too.
struct DeviceGuard {
  int prev = -1, want;
  explicit DeviceGuard(int d) : want(d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) RTS_CUDA(cudaSetDevice(d));
  }
  ~DeviceGuard() {
    if (prev >= 0 && prev != want) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

// Status of an exception caught at the C boundary: the code an rts::Error
// carries, RTS_ERR_NOMEM for a failed host allocation, RTS_ERR_STATE else.
inline rts_status status_of(const std::exception &e) {
  if (const auto *r = dynamic_cast<const Error *>(&e)) return r->code;
  if (dynamic_cast<const std::bad_alloc *>(&e)) return RTS_ERR_NOMEM;
  return RTS_ERR_STATE;
}

// Record `msg` as the calling thread's last error (rts_last_error(NULL)).
rts_status set_thread_error(rts_status code, const std::string &msg);

inline uint64_t words_for(uint64_t nrows) { return (nrows + 31) >> 5; }

// One term of a fused launch: hit iff (x - lo) <= span, unsigned, which is
// lo <= x <= hi for span = hi - lo.
struct DevTerm {
  const uint32_t *col;
  uint32_t lo;
  uint32_t span;
};

struct ScanParams {
  DevTerm t[kFusedMaxTerms];
  int nterms;
  int and_into;  // 1: AND the result into the words already in `out`
  uint32_t *out;
  unsigned long long *count;  // may be null
  uint64_t nrows;
  uint64_t full_tiles;        // tiles of kTileRows rows entirely below nrows
};

// ---- kernel launchers (scan_kernels.cu) ----
struct LaunchShape {
  int blocks;
  int threads;
};
void launch_scan_fused(const ScanParams &p, bool vector_ok, int sm_count, cudaStream_t s);
void launch_bitmap_op(int op, uint32_t *dst, const uint32_t *a, const uint32_t *b, uint64_t words,
                      uint32_t value, int sm_count, cudaStream_t s);
void launch_bitmap_count(const uint32_t *bm, uint64_t nbits, unsigned long long *count, int sm_count,
                         cudaStream_t s);
// Loads onto the current device every kernel that a separate-pass scan of
// single-term passes launches (fused one-term scans, aligned or not, the
// bitmap AND, the count, the fill), which CUDA's lazy module loading would
// otherwise load, allocating device memory, at their first launch.
cudaError_t preload_separate_scan_kernels();
void launch_fill_range(uint32_t *out, uint64_t nrows, bool ones, unsigned long long *count,
                       int sm_count, cudaStream_t s);
// counts[slots[i]] = 0 for i < n, in one launch per 512 slots.
void launch_zero_counts(unsigned long long *counts, const int32_t *slots, int n, cudaStream_t s);
// base[offs[i]] = value for i < n, in one launch per 512 words.
void launch_set_words(uint32_t *base, const uint32_t *offs, int n, uint32_t value, cudaStream_t s);

// ---- BinDex on the GPU (bindex.cu) ----
struct GpuBinDex {
  int K = 0;
  uint64_t n = 0;
  uint32_t *sval = nullptr;   // values in sorted order (n)
  uint32_t *spos = nullptr;   // row of each sorted value (n)
  uint32_t *fv = nullptr;     // (K-1) filter vectors of words_for(n) words each
  uint64_t fv_stride = 0;     // words per filter vector (>= words_for(n), multiple of 4)
  std::vector<uint32_t> start;      // area start values (K), host copy
  std::vector<uint64_t> first_rank; // lower_bound of start[k] in sorted order (K), host copy
  std::vector<uint32_t> sample;     // every kSampleStride-th sorted value, host copy
  uint32_t min_val = 0, max_val = 0;
  ~GpuBinDex();
};
constexpr int kSampleStride = 1024;
struct QuerySlot;                 // context memory of one BinDex query launch (bindex.cu)
constexpr int kQuerySlots = 64;
// Filter-vector words of an index (K start values on the device, K-1
// vectors of fv_stride words) that differ from the ones the start values
// give for the column: 0 for a consistent index.  Synchronises stream s.
uint64_t count_fv_mismatches(const uint32_t *col, uint64_t n, const uint32_t *d_start, int K, const uint32_t *fv,
                             uint64_t fv_stride, unsigned long long *d_bad, int sm_count, cudaStream_t s);
std::unique_ptr<GpuBinDex> build_bindex(const uint32_t *col, uint64_t n, int K, int sm_count,
                                        cudaStream_t s);
// Conjunctive query through the column indexes (all referenced columns
// must be indexed).  Throws rts::Error.
void bindex_query(rts_ctx *ctx, const rts_term *terms, int nterms, uint32_t *out, unsigned long long *count,
                  cudaStream_t s);

// Rank encoding of the resident table (encode.cu): per column the sorted
// original values (the value -> code map), and the code of rank r is
// min + r * step.
struct EncodeMap {
  uint64_t n = 0;
  uint32_t min = 0, step = 1;
  std::vector<uint32_t *> sval;
  ~EncodeMap();
};

// A 256-byte device buffer owned by the context (blocking-call counts).
unsigned long long *small_device_buffer(rts_ctx *ctx);

// ---- batched scan (batch.cu) ----
struct BatchScratch;
void destroy_batch(BatchScratch *b);
struct HostBatchBuffers;
void destroy_host_batch(HostBatchBuffers *b);
// Launch shape of the batched kernels: the variant, warps per CTA (variant
// 3: 8 or 16), queries per pass (<= 512 for variant 4, <= 256 for 3) and the
// shared-memory bytes a pass may spend on its mask tables (the rest of the
// CTA's shared memory stages result words and row positions).
struct BatchConfig {
  int variant = 4;                // 4: passes of up to 512 queries over CTA-wide blocks; 3: 256-query passes per warp
  int warps_per_cta = 16;         // variant 3 only
  int max_queries_per_pass = 512;
  size_t table_budget = 136 * 1024;
};
void batch_scan(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int nq, uint32_t *out,
                uint64_t stride_words, unsigned long long *counts, cudaStream_t s, size_t table_budget);

}  // namespace rts

// The context.  Defined here so every translation unit sees one layout.
struct rts_ctx {
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  uint64_t nrows = 0;
  std::vector<const uint32_t *> cols;
  uint32_t *owned = nullptr;  // one allocation backing owned columns
  size_t owned_bytes = 0;     // its size
  uint64_t col_stride = 0;    // values between owned columns
  std::vector<std::unique_ptr<rts::GpuBinDex>> bindex;
  // scratch for the separate-pass path and the BinDex planner
  std::vector<uint32_t *> scratch_bm;
  uint64_t scratch_words = 0;
  void *plan_dev = nullptr;
  size_t plan_bytes = 0;
  void *plan_host = nullptr;  // pinned
  void *small_dev = nullptr;
  rts::QuerySlot *query_slots = nullptr;  // BinDex query launches (rts::kQuerySlots, used in turn)
  uint64_t query_next = 0;
  void *agg_dev = nullptr;    // compaction scratch (tile counts and offsets)
  size_t agg_bytes = 0;
  rts::BatchScratch *batch = nullptr;
  rts::HostBatchBuffers *host_batch = nullptr;
  rts::BatchConfig batch_cfg;
  std::string tune_report;  // JSON of the last rts_autotune_batch (rts_autotune_report)
  std::unique_ptr<rts::EncodeMap> encode;  // set by rts_encode_table
  std::atomic<uint64_t> launches{0};
  std::string err;
  ~rts_ctx();
};
