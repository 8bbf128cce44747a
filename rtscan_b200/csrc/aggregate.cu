// After the scan: result bitmaps to row ids, masked sums, and a fused
// scan-and-aggregate.
//
// The reference stops at the bitmap and its hit count; its query files name
// the step that follows in a query engine -- TPC-H Q6, a filtered sum of
// l_extendedprice * l_discount (test/scan_cmd_1e8-1c.txt:48-54).  These
// kernels are HBM-bound streaming passes:
//
//   * rts_bitmap_rows_async: ordered compaction of a bitmap into ascending
//     uint32 row ids.  Pass 1 counts the set bits of each 4096-word tile;
//     one CTA turns the tile counts into output offsets; pass 2 reloads each
//     tile into shared memory and every thread expands its 16 consecutive
//     words at its exclusive prefix.  Bytes: 2 x N/8 read + 4 per row id.
//   * rts_bitmap_sum_async: sum of a column, or of the product of two
//     columns, over the set rows (128-bit exact).  A warp takes 1024 rows:
//     its 32 bitmap words, then the values as 16-byte loads, each lane
//     fetching its four rows' bits from the owning lane.  Bytes: N/8 + 4·N
//     per column.
//   * rts_scan_aggregate_async: the conjunctive predicate and the sum in one
//     pass with no bitmap: terms are merged per column into one inclusive
//     range, a thread tests four rows per 16-byte load of every referenced
//     column once, and accumulates the count and the sum.  Bytes: 4·N per
//     referenced column (a column used by the predicate and the sum is read
//     once).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "rts_internal.h"

namespace rts {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kCompactThreads = 256;
constexpr int kCompactWordsPerThread = 16;
constexpr int kCompactTileWords = kCompactThreads * kCompactWordsPerThread;  // 4096 words = 131072 rows
constexpr int kScanThreads = 1024;

// Bitmap words of tile t, padded so that thread i's 16 consecutive words sit
// in 16 different banks from its neighbours' (index w + w/16).
__device__ __forceinline__ int pad16(int w) { return w + (w >> 4); }

__global__ void __launch_bounds__(kCompactThreads) compact_count_kernel(const uint32_t *__restrict__ bm,
                                                                        uint64_t words, uint32_t tail_mask,
                                                                        uint32_t *__restrict__ tile_count) {
  const uint64_t w0 = (uint64_t)blockIdx.x * kCompactTileWords;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < kCompactWordsPerThread; j++) {
    const uint64_t w = w0 + j * kCompactThreads + threadIdx.x;
    if (w < words) c += __popc(w + 1 == words ? bm[w] & tail_mask : bm[w]);
  }
  c = __reduce_add_sync(kFull, c);
  __shared__ uint32_t part[kCompactThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint32_t v = threadIdx.x < kCompactThreads / 32 ? part[threadIdx.x] : 0u;
    v = __reduce_add_sync(kFull, v);
    if (threadIdx.x == 0) tile_count[blockIdx.x] = v;
  }
}

// One CTA: exclusive prefix of the tile counts (as uint64) and the total.
__global__ void __launch_bounds__(kScanThreads) compact_scan_kernel(const uint32_t *__restrict__ tile_count,
                                                                    uint64_t ntiles,
                                                                    unsigned long long *__restrict__ tile_off,
                                                                    unsigned long long *__restrict__ total) {
  const uint64_t per = (ntiles + kScanThreads - 1) / kScanThreads;
  const uint64_t b = threadIdx.x * per, e = std::min<uint64_t>(ntiles, b + per);
  unsigned long long s = 0;
  for (uint64_t i = b; i < e; i++) s += tile_count[i];
  // block-wide inclusive scan of the thread sums
  __shared__ unsigned long long warp_sum[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned long long v = warp_sum[lane], vi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(kFull, vi, o);
      if (lane >= o) vi += y;
    }
    warp_sum[lane] = vi - v;  // exclusive prefix of the warp sums
  }
  __syncthreads();
  unsigned long long off = warp_sum[warp] + incl - s;
  for (uint64_t i = b; i < e; i++) {
    tile_off[i] = off;
    off += tile_count[i];
  }
  if (threadIdx.x == kScanThreads - 1) *total = off;
}

__global__ void __launch_bounds__(kCompactThreads) compact_write_kernel(
    const uint32_t *__restrict__ bm, uint64_t words, uint32_t tail_mask,
    const unsigned long long *__restrict__ tile_off, uint32_t *__restrict__ rows, uint64_t capacity) {
  __shared__ uint32_t tile[kCompactTileWords + kCompactTileWords / 16];
  __shared__ uint32_t warp_sum[kCompactThreads / 32];
  const uint64_t w0 = (uint64_t)blockIdx.x * kCompactTileWords;
#pragma unroll
  for (int j = 0; j < kCompactWordsPerThread; j++) {
    const int i = j * kCompactThreads + threadIdx.x;
    const uint64_t w = w0 + i;
    tile[pad16(i)] = w < words ? (w + 1 == words ? bm[w] & tail_mask : bm[w]) : 0u;
  }
  __syncthreads();
  uint32_t mine[kCompactWordsPerThread];
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < kCompactWordsPerThread; j++) {
    mine[j] = tile[pad16(threadIdx.x * kCompactWordsPerThread + j)];
    c += __popc(mine[j]);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int k = 0; k < warp; k++) before += warp_sum[k];
  unsigned long long o = tile_off[blockIdx.x] + before + incl - c;
  const uint64_t row0 = (w0 + (uint64_t)threadIdx.x * kCompactWordsPerThread) * 32;
#pragma unroll
  for (int j = 0; j < kCompactWordsPerThread; j++) {
    uint32_t w = mine[j];
    while (w) {  // MSB-first: bit 31 is the word's first row
      const int b = __clz(w);
      if (o < capacity) rows[o] = (uint32_t)(row0 + j * 32 + b);
      o++;
      w &= ~(0x80000000u >> b);
    }
  }
}

// 128-bit accumulation: per-thread unsigned __int128, one pair of 64-bit
// atomics per CTA with the carry of the low half propagated.
__device__ __forceinline__ void add128(unsigned long long *res, unsigned __int128 v) {
  const unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
  const unsigned long long old = atomicAdd(res, lo);
  const unsigned long long carry = old + lo < old ? 1ull : 0ull;
  if (hi + carry) atomicAdd(res + 1, hi + carry);
}

__device__ __forceinline__ unsigned __int128 block_sum128(unsigned __int128 v) {
  __shared__ unsigned long long part[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long l2 = __shfl_xor_sync(kFull, lo, o), h2 = __shfl_xor_sync(kFull, hi, o);
    const unsigned long long nl = lo + l2;
    hi += h2 + (nl < lo ? 1ull : 0ull);
    lo = nl;
  }
  if (lane == 0) {
    part[0][warp] = lo;
    part[1][warp] = hi;
  }
  __syncthreads();
  unsigned __int128 t = 0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += ((unsigned __int128)part[1][k] << 64) | part[0][k];
  return t;
}

// Sum of a (or a * b when b) over the set rows of bm; a warp takes 1024 rows.
template <bool PRODUCT>
__global__ void __launch_bounds__(256) bitmap_sum_kernel(const uint32_t *__restrict__ bm, const uint32_t *__restrict__ a,
                                                         const uint32_t *__restrict__ b, uint64_t nrows, int vec,
                                                         unsigned long long *__restrict__ res) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t ntiles = (nrows + 1023) / 1024, words = (nrows + 31) >> 5;
  unsigned __int128 acc = 0;
  for (uint64_t t = warp; t < ntiles; t += nwarps) {
    const uint64_t wi = t * 32 + lane;
    uint32_t myword = wi < words ? bm[wi] : 0u;
    if (wi + 1 == words && (nrows & 31)) myword &= ~(0xFFFFFFFFu >> (nrows & 31));  // bits past nrows
    const uint64_t row0 = t * 1024;
    const bool full = vec && row0 + 1024 <= nrows;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint32_t w = __shfl_sync(kFull, myword, j * 4 + (lane >> 3));
      const uint64_t r = row0 + j * 128 + lane * 4;
      uint32_t va[4], vb[4] = {1u, 1u, 1u, 1u};
      if (full) {
        const uint4 x = *reinterpret_cast<const uint4 *>(a + r);
        va[0] = x.x, va[1] = x.y, va[2] = x.z, va[3] = x.w;
        if (PRODUCT) {
          const uint4 y = *reinterpret_cast<const uint4 *>(b + r);
          vb[0] = y.x, vb[1] = y.y, vb[2] = y.z, vb[3] = y.w;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 4; k++) {
          va[k] = r + k < nrows ? a[r + k] : 0u;
          if (PRODUCT) vb[k] = r + k < nrows ? b[r + k] : 0u;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int bit = 31 - ((lane & 7) * 4 + k);
        if ((w >> bit) & 1u) acc += PRODUCT ? (unsigned __int128)((unsigned long long)va[k] * vb[k]) : va[k];
      }
    }
  }
  const unsigned __int128 t = block_sum128(acc);
  if (threadIdx.x == 0 && t) add128(res, t);
}

// Fused predicate + aggregate.  Column slot 0 is the first aggregate column
// and slot 1 the second (when MODE needs them); every slot carries the
// merged range of the terms on that column ((0, 2^32 - 1) when it has none).
struct AggParams {
  const uint32_t *col[8];
  uint32_t lo[8];
  uint32_t span[8];
  uint64_t nrows;
  unsigned long long *count;  // may be null
  unsigned long long *sum;    // two words (low, high); may be null
};

// MODE 0: count only; 1: sum of slot 0; 2: sum of slot 0 x slot 1;
// 3: sum of slot 0 squared.
template <int NU, int MODE, bool VEC>
__global__ void __launch_bounds__(256) scan_aggregate_kernel(const __grid_constant__ AggParams p) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long cnt = 0;
  unsigned __int128 acc = 0;
  auto one = [&](const uint32_t (&v)[NU]) {
    bool hit = true;
#pragma unroll
    for (int c = 0; c < NU; c++) hit = hit && (v[c] - p.lo[c] <= p.span[c]);
    cnt += hit;
    if (MODE == 1 && hit) acc += v[0];
    if (MODE == 2 && hit) acc += (unsigned __int128)((unsigned long long)v[0] * v[NU > 1 ? 1 : 0]);
    if (MODE == 3 && hit) acc += (unsigned __int128)((unsigned long long)v[0] * v[0]);
  };
  const uint64_t groups = VEC ? p.nrows / 4 : 0;
  for (uint64_t g = tid; g < groups; g += nth) {
    uint4 x[NU];
#pragma unroll
    for (int c = 0; c < NU; c++) x[c] = __ldg(reinterpret_cast<const uint4 *>(p.col[c]) + g);
    uint32_t v[NU];
#pragma unroll
    for (int c = 0; c < NU; c++) v[c] = x[c].x;
    one(v);
#pragma unroll
    for (int c = 0; c < NU; c++) v[c] = x[c].y;
    one(v);
#pragma unroll
    for (int c = 0; c < NU; c++) v[c] = x[c].z;
    one(v);
#pragma unroll
    for (int c = 0; c < NU; c++) v[c] = x[c].w;
    one(v);
  }
  for (uint64_t r = groups * 4 + tid; r < p.nrows; r += nth) {
    uint32_t v[NU];
#pragma unroll
    for (int c = 0; c < NU; c++) v[c] = __ldg(p.col[c] + r);
    one(v);
  }
  if (p.count) {
    unsigned long long c = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(p.count, c);
  }
  if (MODE > 0 && p.sum) {
    const unsigned __int128 t = block_sum128(acc);
    if (threadIdx.x == 0 && t) add128(p.sum, t);
  }
}

template <int NU, int MODE>
void launch_agg(const AggParams &p, bool vec, int sm_count, cudaStream_t s) {
  const uint64_t work = vec ? p.nrows / 4 : p.nrows;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, (uint64_t)sm_count * 8));
  if (vec) scan_aggregate_kernel<NU, MODE, true><<<grid, 256, 0, s>>>(p);
  else scan_aggregate_kernel<NU, MODE, false><<<grid, 256, 0, s>>>(p);
}

template <int MODE>
void launch_agg_nu(int nu, const AggParams &p, bool vec, int sm_count, cudaStream_t s) {
  switch (nu) {
    case 1: launch_agg<1, MODE>(p, vec, sm_count, s); break;
    case 2: launch_agg<2, MODE>(p, vec, sm_count, s); break;
    case 3: launch_agg<3, MODE>(p, vec, sm_count, s); break;
    case 4: launch_agg<4, MODE>(p, vec, sm_count, s); break;
    case 5: launch_agg<5, MODE>(p, vec, sm_count, s); break;
    case 6: launch_agg<6, MODE>(p, vec, sm_count, s); break;
    case 7: launch_agg<7, MODE>(p, vec, sm_count, s); break;
    default: launch_agg<8, MODE>(p, vec, sm_count, s); break;
  }
}

// Device scratch for the compaction's tile counts and offsets (grown as needed).
void *agg_scratch(rts_ctx *ctx, size_t bytes) {
  if (ctx->agg_bytes < bytes) {
    if (ctx->agg_dev) cudaFree(ctx->agg_dev);
    ctx->agg_dev = nullptr;
    ctx->agg_bytes = 0;
    if (cudaMalloc(&ctx->agg_dev, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "aggregate scratch allocation failed");
    }
    ctx->agg_bytes = bytes;
  }
  return ctx->agg_dev;
}


rts_status fail(rts_ctx *ctx, const std::exception &e) {
  if (ctx) ctx->err = e.what();
  return set_thread_error(status_of(e), e.what());
}

}  // namespace
}  // namespace rts

extern "C" {

rts_status rts_bitmap_rows_async(rts_ctx *ctx, const uint32_t *dev_bitmap, uint64_t nrows, uint32_t *dev_rows,
                                 uint64_t capacity, uint64_t *dev_count, void *stream) {
  rts::Range nvtx_range_("rts_bitmap_rows_async");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!dev_bitmap || !dev_count || (capacity && !dev_rows)) throw rts::Error(RTS_ERR_ARG, "null argument");
    if (nrows > 0xFFFFFFFFull) throw rts::Error(RTS_ERR_ARG, "row ids are uint32: at most 2^32 - 1 rows");
    rts::DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t words = rts::words_for(nrows);
    if (words == 0) {
      RTS_CUDA(cudaMemsetAsync(dev_count, 0, 8, s));
      return RTS_OK;
    }
    const uint32_t tail_mask = (nrows & 31) ? ~(0xFFFFFFFFu >> (nrows & 31)) : 0xFFFFFFFFu;
    const uint64_t ntiles = (words + rts::kCompactTileWords - 1) / rts::kCompactTileWords;
    char *scratch = static_cast<char *>(rts::agg_scratch(ctx, ntiles * 12 + 16));
    auto *tile_off = reinterpret_cast<unsigned long long *>(scratch);
    auto *tile_count = reinterpret_cast<uint32_t *>(scratch + ntiles * 8);
    rts::compact_count_kernel<<<(unsigned)ntiles, rts::kCompactThreads, 0, s>>>(dev_bitmap, words, tail_mask,
                                                                               tile_count);
    rts::compact_scan_kernel<<<1, rts::kScanThreads, 0, s>>>(tile_count, ntiles, tile_off,
                                                             reinterpret_cast<unsigned long long *>(dev_count));
    rts::compact_write_kernel<<<(unsigned)ntiles, rts::kCompactThreads, 0, s>>>(dev_bitmap, words, tail_mask,
                                                                               tile_off, dev_rows, capacity);
    RTS_CUDA(cudaGetLastError());
    ctx->launches += 3;
    return RTS_OK;
  } catch (const std::exception &e) {
    return rts::fail(ctx, e);
  }
}

rts_status rts_bitmap_sum_async(rts_ctx *ctx, const uint32_t *dev_bitmap, int32_t col_a, int32_t col_b,
                                uint64_t *dev_sum, void *stream) {
  rts::Range nvtx_range_("rts_bitmap_sum_async");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!dev_bitmap || !dev_sum) throw rts::Error(RTS_ERR_ARG, "null argument");
    const int nc = (int)ctx->cols.size();
    if (col_a < 0 || col_a >= nc || col_b < -1 || col_b >= nc) throw rts::Error(RTS_ERR_ARG, "column out of range");
    rts::DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t *a = ctx->cols[col_a], *b = col_b >= 0 ? ctx->cols[col_b] : nullptr;
    const bool vec = (((uintptr_t)a | (uintptr_t)(b ? b : a)) & 15) == 0;
    const uint64_t ntiles = (ctx->nrows + 1023) / 1024;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((ntiles + 7) / 8, (uint64_t)ctx->sm_count * 8));
    RTS_CUDA(cudaMemsetAsync(dev_sum, 0, 16, s));
    auto *res = reinterpret_cast<unsigned long long *>(dev_sum);
    if (b) rts::bitmap_sum_kernel<true><<<grid, 256, 0, s>>>(dev_bitmap, a, b, ctx->nrows, vec ? 1 : 0, res);
    else rts::bitmap_sum_kernel<false><<<grid, 256, 0, s>>>(dev_bitmap, a, nullptr, ctx->nrows, vec ? 1 : 0, res);
    RTS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return RTS_OK;
  } catch (const std::exception &e) {
    return rts::fail(ctx, e);
  }
}

rts_status rts_scan_aggregate_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, int32_t col_a,
                                    int32_t col_b, uint64_t *dev_count, uint64_t *dev_sum, void *stream) {
  rts::Range nvtx_range_("rts_scan_aggregate_async");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (nterms < 0 || (nterms > 0 && !terms)) throw rts::Error(RTS_ERR_ARG, "bad terms");
    const int nc = (int)ctx->cols.size();
    if (nc == 0) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (col_a < -1 || col_a >= nc || col_b < -1 || col_b >= nc || (col_b >= 0 && col_a < 0))
      throw rts::Error(RTS_ERR_ARG, "aggregate column out of range");
    if (col_a >= 0 && !dev_sum) throw rts::Error(RTS_ERR_ARG, "a sum needs dev_sum");
    // slots: aggregate columns first, then the predicate's other columns
    std::vector<int> slot_col;
    std::vector<uint32_t> lo, hi;
    auto slot_of = [&](int col) {
      for (size_t i = 0; i < slot_col.size(); i++)
        if (slot_col[i] == col) return (int)i;
      slot_col.push_back(col);
      lo.push_back(0);
      hi.push_back(0xFFFFFFFFu);
      return (int)slot_col.size() - 1;
    };
    if (col_a >= 0) slot_of(col_a);
    if (col_b >= 0 && col_b != col_a) slot_of(col_b);
    bool empty = false;
    for (int i = 0; i < nterms; i++) {
      const rts_term &t = terms[i];
      if (t.column < 0 || t.column >= nc) throw rts::Error(RTS_ERR_ARG, "term column out of range");
      if (t.lo > t.hi) empty = true;
      const int k = slot_of(t.column);
      lo[k] = std::max(lo[k], t.lo);
      hi[k] = std::min(hi[k], t.hi);
      if (lo[k] > hi[k]) empty = true;
    }
    if (slot_col.size() > 8) throw rts::Error(RTS_ERR_ARG, "at most 8 distinct columns per aggregate scan");
    rts::DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (dev_count) RTS_CUDA(cudaMemsetAsync(dev_count, 0, 8, s));
    if (dev_sum) RTS_CUDA(cudaMemsetAsync(dev_sum, 0, 16, s));
    if (empty || ctx->nrows == 0) return RTS_OK;
    if (slot_col.empty()) slot_of(0);  // no term and no aggregate: count every row
    rts::AggParams p{};
    bool vec = true;
    for (size_t i = 0; i < slot_col.size(); i++) {
      p.col[i] = ctx->cols[slot_col[i]];
      p.lo[i] = lo[i];
      p.span[i] = hi[i] - lo[i];
      vec = vec && ((uintptr_t)p.col[i] & 15) == 0;
    }
    p.nrows = ctx->nrows;
    p.count = reinterpret_cast<unsigned long long *>(dev_count);
    p.sum = reinterpret_cast<unsigned long long *>(dev_sum);
    const int nu = (int)slot_col.size();
    if (col_a < 0) {
      rts::launch_agg_nu<0>(nu, p, vec, ctx->sm_count, s);
    } else if (col_b < 0) {
      rts::launch_agg_nu<1>(nu, p, vec, ctx->sm_count, s);
    } else if (col_b == col_a) {
      rts::launch_agg_nu<3>(nu, p, vec, ctx->sm_count, s);
    } else {
      rts::launch_agg_nu<2>(nu, p, vec, ctx->sm_count, s);
    }
    RTS_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return RTS_OK;
  } catch (const std::exception &e) {
    return rts::fail(ctx, e);
  }
}

}  // extern "C"
