// Allocation-free variant of the separate-pass conjunctive scan.
//
// rts_scan_separate_async keeps one scratch bitmap per context, allocated
// with cudaMalloc on first use.  Some callers cannot let a library allocate
// device memory: an engine that reserves all of HBM for its own pool
// allocator at start-up (a cudaMalloc from the library would then fail or
// eat into memory the engine has promised elsewhere), or a caller on a
// latency-critical path, where cudaMalloc's implicit device-wide
// synchronisation would stall every other stream.  For them this entry
// point takes plain device pointers (no context) and keeps its scratch
// bitmap in a fixed file-scope __device__ array.
//
// The CUDA runtime loads device code lazily: the array (16 MiB) and the
// kernels this entry point launches are placed on a device, in memory the
// runtime allocates, when the first call on that device sets up (it looks
// up the array's address and loads the kernels).  From then on the device
// holds them until the process exits and no call allocates.  A caller that
// will later hand all of HBM to its own pool therefore makes one warm-up
// call per device before reserving the pool (and before any stream
// capture).  A set-up that fails, for instance because the device is
// already full, is reported and retried by the next call.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "rts_internal.h"

namespace {

// Scratch for one predicate pass: RTS_NOALLOC_MAX_ROWS / 32 words (16 MiB).
constexpr uint64_t kScratchWords = RTS_NOALLOC_MAX_ROWS / 32;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
struct DeviceSetup {
  std::mutex mu;
  std::atomic<bool> ready{false};
  uint32_t *scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int sm_count = 0;
};
DeviceSetup g_setup[kMaxDevices];

// Set-up of the current device `dev`, done by its first successful call:
// the device address of the scratch array (its host-side name is not a
// device address), the SM count used to size grids, and the kernels the
// scan launches loaded onto the device.  Nothing is recorded on failure.
cudaError_t setup_for(int dev, DeviceSetup *&out) {
  DeviceSetup &d = g_setup[dev];
  out = &d;
  if (d.ready.load(std::memory_order_acquire)) return cudaSuccess;
  std::lock_guard<std::mutex> lk(d.mu);
  if (d.ready.load(std::memory_order_relaxed)) return cudaSuccess;
  void *p = nullptr;
  int sms = 0;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = rts::preload_separate_scan_kernels();
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear it: the next call tries again
    return e;
  }
  d.scratch = static_cast<uint32_t *>(p);
  d.sm_count = sms;
  d.ready.store(true, std::memory_order_release);
  return cudaSuccess;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

rts_status scan_separate_noalloc(const uint32_t *const *dev_cols, int32_t ncols, uint64_t nrows,
                                 const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap, uint64_t *dev_count,
                                 void *stream) {
  using rts::set_thread_error;
  if (nrows > RTS_NOALLOC_MAX_ROWS)
    return set_thread_error(RTS_ERR_ARG, "nrows " + std::to_string(nrows) +
                                             " exceeds the allocation-free scan's limit of " +
                                             std::to_string((unsigned long long)RTS_NOALLOC_MAX_ROWS) + " rows");
  if (!dev_cols || ncols < 1 || nrows == 0 || !dev_bitmap || !dev_count)
    return set_thread_error(RTS_ERR_ARG, "need device columns, nrows >= 1, a result bitmap and a count");
  if (nterms < 0 || (nterms > 0 && !terms)) return set_thread_error(RTS_ERR_ARG, "bad term list");
  for (int c = 0; c < ncols; c++)
    if (!dev_cols[c]) return set_thread_error(RTS_ERR_ARG, "null column pointer");
  // Group terms per column, intersect their ranges, drop always-true ones.
  std::vector<int> order;
  std::vector<uint32_t> lo, hi;
  bool empty = false;
  for (int i = 0; i < nterms; i++) {
    const rts_term &t = terms[i];
    if (t.column < 0 || t.column >= ncols) return set_thread_error(RTS_ERR_ARG, "term column out of range");
    if (t.lo > t.hi) empty = true;
    auto it = std::find(order.begin(), order.end(), (int)t.column);
    if (it == order.end()) {
      order.push_back(t.column);
      lo.push_back(t.lo);
      hi.push_back(t.hi);
    } else {
      const size_t k = it - order.begin();
      lo[k] = std::max(lo[k], t.lo);
      hi[k] = std::min(hi[k], t.hi);
      if (lo[k] > hi[k]) empty = true;
    }
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_thread_error(RTS_ERR_NODEV, "no current CUDA device");
  DeviceSetup *dp = nullptr;
  e = setup_for(dev, dp);
  if (e != cudaSuccess)
    return set_thread_error(RTS_ERR_CUDA, std::string("set-up of the scratch array and kernels on device ") +
                                              std::to_string(dev) + ": " + cudaGetErrorString(e));
  DeviceSetup &d = *dp;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long *count = reinterpret_cast<unsigned long long *>(dev_count);
  const uint64_t words = rts::words_for(nrows);
  std::vector<rts::DevTerm> live;
  for (size_t k = 0; k < order.size() && !empty; k++)
    if (!(lo[k] == 0 && hi[k] == 0xFFFFFFFFu)) live.push_back({dev_cols[order[k]], lo[k], hi[k] - lo[k]});
  if (empty || live.empty()) {
    rts::launch_fill_range(dev_bitmap, nrows, !empty, count, d.sm_count, s);
  } else {
    // Pass 1 writes the result bitmap; every later pass writes the scratch
    // bitmap, which it overwrites completely before the AND reads it, so
    // nothing left in the array by an earlier call is ever read.
    for (size_t i = 0; i < live.size(); i++) {
      rts::ScanParams p;
      memset(&p, 0, sizeof p);
      p.t[0] = live[i];
      p.nterms = 1;
      p.out = i == 0 ? dev_bitmap : d.scratch;
      p.nrows = nrows;
      p.full_tiles = nrows / rts::kTileRows;
      rts::launch_scan_fused(p, aligned16(p.t[0].col), d.sm_count, s);
      if (i > 0) rts::launch_bitmap_op(RTS_BM_AND, dev_bitmap, dev_bitmap, d.scratch, words, 0, d.sm_count, s);
    }
    e = cudaMemsetAsync(count, 0, 8, s);
    if (e != cudaSuccess) return set_thread_error(RTS_ERR_CUDA, std::string("count reset: ") + cudaGetErrorString(e));
    rts::launch_bitmap_count(dev_bitmap, nrows, count, d.sm_count, s);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_thread_error(RTS_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return RTS_OK;
}

}  // namespace

extern "C" rts_status rts_scan_separate_noalloc_async(const uint32_t *const *dev_cols, int32_t ncols, uint64_t nrows,
                                                      const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap,
                                                      uint64_t *dev_count, void *stream) {
  rts::Range nvtx_range_("rts_scan_separate_noalloc_async");
  try {  // the checks and the plan use host memory only; a failed host allocation is a status
    return scan_separate_noalloc(dev_cols, ncols, nrows, terms, nterms, dev_bitmap, dev_count, stream);
  } catch (const std::exception &e) {
    return rts::set_thread_error(rts::status_of(e), e.what());
  }
}
