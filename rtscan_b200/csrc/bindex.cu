// BinDex on the GPU: index build, sieve, refine.
//
// The reference's BinDex (bindex.cpp:599-671, bindex_cuda.cpp:164-282) sorts
// a column, cuts the sorted order into K equal-count areas (start value of
// area k = sorted[k*(n/K)], duplicate rule bindex.cpp:613-631) and stores
// K-1 filter vectors fv[k] = (x < start value of area k+1) in MSB-first
// order (set_fv_val_less, bindex.cpp:553-560).  A bound "x < b" is answered
// by the filter vector nearest to b plus an XOR refine of the rows between
// that vector's boundary and b (bindex_scan_lt, bindex.cpp:1365-1417).
//
// Here the sorted values and row ids stay in HBM as flat arrays (no
// reference-style 3276-row blocks: on a GPU the refine set of a bound is one
// contiguous range of the sorted order, [lower_bound(S), lower_bound(b))),
// and a conjunctive query runs as two launches:
//   1. sieve: per 32-row word, AND over terms of (U_t & ~L_t), where U_t / L_t
//      are the filter vectors (or constants) nearest to the term's upper and
//      lower bound; popcount into the result count.
//   2. refine: every row of every refine range (rows whose sieve bit may be
//      wrong) is re-tested on all terms with gathered column values and its
//      bit set or cleared with an atomic; the count moves by the number of
//      bits that actually changed.  This is the reference's GPU refine
//      (refineBlock, cuda_and.cu:75-99: test every column's box, then
//      atomicOr / atomicAnd) done in one launch for all ranges instead of
//      one launch per 4096-row block.
// The exact range ends (lower_bound of each bound in the sorted values) are
// found inside the refine kernel by warp-cooperative searches in a window
// the host narrows with a sample of the sorted order, so the host never
// waits for the device.  When one term matches few rows, the planner skips
// the sieve (result starts at zero) and refines that term's match range
// instead (the reference's "one face" case, bindex_cuda.cpp:1533-1567).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "rts_internal.h"

namespace rts {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kThreads = 256;
constexpr int kMaxBounds = 2 * kFusedMaxTerms;
constexpr uint64_t kRefineInSieveRows = 1024;  // estimated refine rows the sieve's last block takes

// First index i in [lo, hi) with a[i] >= b, else hi (a sorted ascending).
// Called by a whole warp; every lane returns the same value.
__device__ uint64_t warp_lower_bound(const uint32_t *a, uint64_t lo, uint64_t hi, uint32_t b) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t idx = lo + (uint64_t)lane * step;
    const bool ge = idx < hi ? (a[idx] >= b) : true;
    const unsigned m = __ballot_sync(kFull, ge);
    if (m == 0) {
      lo = lo + 31 * step + 1;
    } else {
      const int f = __ffs(m) - 1;
      if (f == 0) return lo;
      const uint64_t nlo = lo + (uint64_t)(f - 1) * step + 1;
      const uint64_t nhi = min(lo + (uint64_t)f * step, hi);
      lo = nlo;
      hi = nhi;
    }
  }
  const uint64_t idx = lo + lane;
  const bool ge = idx < hi ? (a[idx] >= b) : false;
  const unsigned m = __ballot_sync(kFull, ge);
  return m ? lo + (uint64_t)(__ffs(m) - 1) : hi;
}

// ---- build -------------------------------------------------------------------

__global__ void iota_kernel(uint32_t *p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

// Area k starts at sorted index k*avg (area 0 at 0); its start value and
// the lower bound of that value in the sorted order.  One warp per area.
__global__ void area_kernel(const uint32_t *sval, uint64_t n, int K, uint32_t *start, unsigned long long *first_rank) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= K) return;
  const uint64_t avg = n / (uint64_t)K;
  const uint32_t v = sval[(uint64_t)warp * avg];
  const uint64_t r = warp_lower_bound(sval, 0, n, v);
  if ((threadIdx.x & 31) == 0) {
    start[warp] = v;
    first_rank[warp] = r;
  }
}

__global__ void sample_kernel(const uint32_t *sval, uint64_t n, uint32_t *out, uint64_t m, uint64_t stride) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x)
    out[j] = sval[j * stride];
}

// fv[k] word w: bit 31-r set iff row 32w+r < n and col[32w+r] < S[k+1].
// A thread owns one word; a(x) = #{i in 1..K-1 : S[i] <= x} is found by a
// binary search over the start values in shared memory, and fv[k] holds the
// rows with a(x) <= k.  A (uint8_t for K <= 256, else uint16_t) holds a(x);
// its largest value marks the padding rows past n, which no fv[k] holds.
// With kCheck the words are compared with fv instead of written and the
// mismatching words counted into *bad (an index loaded from a file).
template <typename A, bool kCheck>
__global__ void __launch_bounds__(kThreads) fv_kernel(const uint32_t *col, uint64_t n, const uint32_t *start, int K,
                                                      uint32_t *fv, uint64_t fv_stride, unsigned long long *bad) {
  extern __shared__ uint32_t s_start[];
  for (int i = threadIdx.x; i < K; i += blockDim.x) s_start[i] = start[i];
  __syncthreads();
  const uint64_t words = (n + 31) >> 5;
  unsigned long long b = 0;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
    A a[32];
    const uint64_t row0 = w * 32;
#pragma unroll
    for (int r = 0; r < 32; r++) {
      const uint64_t row = row0 + r;
      if (row < n) {
        const uint32_t x = col[row];
        int lo = 1, hi = K;  // first i in [1, K) with S[i] > x
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (s_start[mid] <= x) lo = mid + 1; else hi = mid;
        }
        a[r] = (A)(lo - 1);
      } else {
        a[r] = (A)~A(0);
      }
    }
    for (int k = 0; k < K - 1; k++) {
      uint32_t word = 0;
#pragma unroll
      for (int r = 0; r < 32; r++) word |= (a[r] <= k ? 1u : 0u) << (31 - r);
      if (kCheck) b += fv[(uint64_t)k * fv_stride + w] != word;
      else fv[(uint64_t)k * fv_stride + w] = word;
    }
  }
  if (kCheck) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(kFull, b, o);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(bad, b);
  }
}

int blocks_for(uint64_t items, int sm_count, int per_sm);

template <bool kCheck>
void launch_fv(const uint32_t *col, uint64_t n, const uint32_t *start, int K, uint32_t *fv, uint64_t fv_stride,
               unsigned long long *bad, int sm_count, cudaStream_t s) {
  const uint64_t words = (n + 31) >> 5;
  if (K <= 256)
    fv_kernel<uint8_t, kCheck><<<blocks_for(words, sm_count, 8), kThreads, K * sizeof(uint32_t), s>>>(
        col, n, start, K, fv, fv_stride, bad);
  else
    fv_kernel<uint16_t, kCheck><<<blocks_for(words, sm_count, 8), kThreads, K * sizeof(uint32_t), s>>>(
        col, n, start, K, fv, fv_stride, bad);
}

// ---- query -------------------------------------------------------------------
//
// A query is two launches on the caller's stream: the sieve kernel writes
// every result word once (U & ~L over terms, or zeros in candidate mode);
// its blocks sum their popcounts into a context slot and the last block to
// finish (an arrival ticket, no waiting) stores the count.  The refine
// kernel, launched as a programmatic dependent of the sieve, resolves the
// refine ranges' ends (warp searches in the sorted values) and tests its
// first rows while the sieve streams, then corrects the rows whose bit the
// sieve got wrong, and the count, with atomics.  Small refine sets are
// re-tested by the sieve's last block instead (its block 0 resolves their
// ends into the slot).

// A refine range end: a known sorted rank, or the lower bound of `b` in the
// sorted values, searched in [wlo, whi].
struct RangeEnd {
  uint64_t rank;  // kind 0
  uint64_t wlo, whi;
  uint32_t b;
  int kind;       // 0 = rank, 1 = lower_bound(b)
};

struct RefineRange {
  const uint32_t *sval;
  const uint32_t *spos;
  RangeEnd e0, e1;
  int term;              // the term on this range's column (its value is sval[i])
  uint32_t wlo, wspan;   // the values of its rows: x - wlo <= wspan (the ends' lower bounds)
  int wok;               // 0: an empty range
};

// The sieve's verdict on one term of a row, as a value range: the filter
// vectors it ANDs are (x < start) bits, so U & ~L holds exactly for
// lo <= x < hi of the chosen areas' start values; ok = 0 when it holds for
// no value.
struct ApproxTerm {
  uint32_t lo, span;
  int ok;
};

}  // namespace

// Context memory shared by the launches of one query (kQuerySlots of them,
// used in turn, so queries on different streams do not share one): the
// refine ranges the sieve's last block re-tests, and the sieve's running
// count and finished blocks, both zero between queries.
struct QuerySlot {
  unsigned long long acc;
  unsigned int ticket;
  unsigned int pad;
  unsigned long long begin[kMaxBounds], end[kMaxBounds];
};

namespace {

struct SieveTerm {
  const uint32_t *U;  // upper-bound approximation (x < b_hi); null = constant
  const uint32_t *L;  // lower-bound approximation (x < b_lo); null = constant
  uint32_t u_const;   // value of U when null (0 or ~0)
  uint32_t l_const;   // value of L when null
};

struct SieveParams {
  SieveTerm t[kFusedMaxTerms];
  int nterms;         // 0: candidate mode, every word zero
  uint32_t *out;
  unsigned long long *count;
  uint64_t words;
  uint32_t tail_mask;  // mask of the last word (rows past n are zero)
  int vec;
  QuerySlot *slot;
  RefineRange r[kMaxBounds];  // the refine ranges whose ends block 0 resolves
  int nranges;
  // small refine sets: the last block to finish (every word written by
  // then) re-tests them here and no refine launch follows
  int refine_here;
  int zero_start;
  DevTerm rt[kFusedMaxTerms];
  ApproxTerm ra[kFusedMaxTerms];
  int rnterms;
};

__device__ __forceinline__ uint32_t sieve_word(const SieveParams &p, uint64_t w) {
  uint32_t r = 0xFFFFFFFFu;
  for (int t = 0; t < p.nterms; t++) {
    const SieveTerm &s = p.t[t];
    const uint32_t u = s.U ? __ldg(s.U + w) : s.u_const;
    const uint32_t l = s.L ? __ldg(s.L + w) : s.l_const;
    r &= u & ~l;
  }
  return p.nterms ? r : 0u;
}

__device__ __forceinline__ uint4 ld4(const uint32_t *p, uint64_t i4) {
  return __ldg(reinterpret_cast<const uint4 *>(p) + i4);
}

__device__ uint64_t resolve_end(const RefineRange &rg, const RangeEnd &e) {
  if (e.kind == 0) return e.rank;
  return warp_lower_bound(rg.sval, e.wlo, e.whi, e.b);
}

// Wait for the grid this one depends on (launched with programmatic stream
// serialization) to complete, its writes visible; returns at once in a grid
// launched without it.
__device__ __forceinline__ void wait_prerequisite() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Re-test the rows of the refine ranges (ends begin[r], end[r]) that fall to
// thread `tid` of `stride`, correct their bits; returns the change of the
// count.  A row's bit as the sieve left it is the AND of the terms'
// ApproxTerm verdicts on its values (zero in candidate mode), its right bit
// the AND of the exact terms, so only rows whose two differ are written,
// with atomics whose old value is not needed.  A row in several ranges
// (the windows of two terms) is corrected and counted by the first of them.
// R rows per iteration: their loads (row id, own value, gathers) are
// issued before any row's test.  kWait: the bits belong to the grid this
// one depends on, so the first atomic waits for it (the loads and tests of
// the first rows before it overlap that grid).
template <bool kWait, int R>
__device__ long long refine_rows(const RefineRange *ranges, int nranges, const DevTerm *terms,
                                 const ApproxTerm *approx, int nterms, const unsigned long long *begin,
                                 const unsigned long long *end, uint64_t tid, uint64_t stride, bool zero_start,
                                 uint32_t *out) {
  long long delta = 0;
  bool waited = !kWait;
  for (int r = 0; r < nranges; r++) {
    const RefineRange &rg = ranges[r];
    const uint64_t e = end[r];
    for (uint64_t i = begin[r] + tid; i < e; i += R * stride) {
      uint32_t row[R];
      int flip[R];  // +1 set, -1 clear, 0 leave
#pragma unroll
      for (int k = 0; k < R; k++) {
        const uint64_t ik = i + k * stride;
        const bool in = ik < e;
        row[k] = in ? __ldg(rg.spos + ik) : 0u;
        const uint32_t own = in ? __ldg(rg.sval + ik) : 0u;
        bool now = true, was = !zero_start, first = in;
        for (int t = 0; t < nterms; t++) {
          const uint32_t x = t == rg.term ? own : __ldg(terms[t].col + row[k]);
          now = now && x - terms[t].lo <= terms[t].span;
          was = was && approx[t].ok && x - approx[t].lo <= approx[t].span;
          for (int q = 0; q < r; q++)
            first = first && !(ranges[q].term == t && ranges[q].wok && x - ranges[q].wlo <= ranges[q].wspan);
        }
        flip[k] = first ? (int)now - (int)was : 0;
      }
#pragma unroll
      for (int k = 0; k < R; k++) {
        if (!flip[k]) continue;
        if (!waited) {
          wait_prerequisite();
          waited = true;
        }
        const uint32_t bit = 1u << (31 - (row[k] & 31));
        uint32_t *word = out + (row[k] >> 5);
        if (flip[k] > 0) atomicOr(word, bit);
        else atomicAnd(word, ~bit);
        delta += flip[k];
      }
    }
  }
  return delta;
}

__global__ void __launch_bounds__(kThreads) sieve_kernel(const __grid_constant__ SieveParams p) {
  // a refine grid launched after this one may start now (see refine_kernel)
  asm volatile("griddepcontrol.launch_dependents;");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (p.refine_here && blockIdx.x == 0) {
    for (int r = warp; r < p.nranges; r += kThreads / 32) {
      const uint64_t a = resolve_end(p.r[r], p.r[r].e0);
      const uint64_t b = resolve_end(p.r[r], p.r[r].e1);
      if (lane == 0) {
        p.slot->begin[r] = min(a, b);
        p.slot->end[r] = max(a, b);
      }
    }
  }
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t cnt = 0;
  uint64_t done = 0;
  if (p.vec) {
    const uint64_t nv = (p.words - 1) / 4;  // vectors entirely before the last word
    // two vectors per iteration: each thread keeps the loads of both in flight
    for (uint64_t i = tid; i < nv; i += 2 * stride) {
      const uint64_t i2 = i + stride;
      const bool two = i2 < nv;
      uint4 r = make_uint4(0, 0, 0, 0), r2 = r;
      if (p.nterms) {
        r = r2 = make_uint4(~0u, ~0u, ~0u, ~0u);
        for (int t = 0; t < p.nterms; t++) {
          const SieveTerm &s = p.t[t];
          const uint4 cu = make_uint4(s.u_const, s.u_const, s.u_const, s.u_const);
          const uint4 cl = make_uint4(s.l_const, s.l_const, s.l_const, s.l_const);
          const uint4 u = s.U ? ld4(s.U, i) : cu;
          const uint4 l = s.L ? ld4(s.L, i) : cl;
          const uint4 u2 = (s.U && two) ? ld4(s.U, i2) : cu;
          const uint4 l2 = (s.L && two) ? ld4(s.L, i2) : cl;
          r.x &= u.x & ~l.x;
          r.y &= u.y & ~l.y;
          r.z &= u.z & ~l.z;
          r.w &= u.w & ~l.w;
          r2.x &= u2.x & ~l2.x;
          r2.y &= u2.y & ~l2.y;
          r2.z &= u2.z & ~l2.z;
          r2.w &= u2.w & ~l2.w;
        }
        cnt += __popc(r.x) + __popc(r.y) + __popc(r.z) + __popc(r.w);
        if (two) cnt += __popc(r2.x) + __popc(r2.y) + __popc(r2.z) + __popc(r2.w);
      }
      reinterpret_cast<uint4 *>(p.out)[i] = r;
      if (two) reinterpret_cast<uint4 *>(p.out)[i2] = r2;
    }
    done = nv * 4;
  }
  for (uint64_t w = done + tid; w < p.words; w += stride) {
    uint32_t r = sieve_word(p, w);
    if (w == p.words - 1) r &= p.tail_mask;
    p.out[w] = r;
    cnt += __popc(r);
  }
  // the block's popcount into the slot; the last block stores the count
  __shared__ unsigned long long part[kThreads / 32];
  cnt = __reduce_add_sync(kFull, cnt);
  if (lane == 0) part[warp] = cnt;
  __syncthreads();
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int i = 0; i < kThreads / 32; i++) s += part[i];
    if (s) atomicAdd(&p.slot->acc, s);
    __threadfence();
    s_last = atomicAdd(&p.slot->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  // the last block: every other block's words and popcount are in place
  __threadfence();
  long long delta = 0;
  if (p.refine_here) {
    __shared__ unsigned long long s_begin[kMaxBounds], s_end[kMaxBounds];
    for (int r = threadIdx.x; r < p.nranges; r += kThreads) {
      s_begin[r] = p.slot->begin[r];
      s_end[r] = p.slot->end[r];
    }
    __syncthreads();
    delta = refine_rows<false, 2>(p.r, p.nranges, p.rt, p.ra, p.rnterms, s_begin, s_end, threadIdx.x, kThreads,
                                  p.zero_start != 0, p.out);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) delta += __shfl_xor_sync(kFull, delta, o);
  __syncthreads();
  if (lane == 0) part[warp] = (unsigned long long)delta;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long d = 0;
    for (int i = 0; i < kThreads / 32; i++) d += (long long)part[i];
    *p.count = atomicExch(&p.slot->acc, 0ull) + (unsigned long long)d;
    p.slot->ticket = 0;
  }
}

struct RefineParams {
  DevTerm t[kFusedMaxTerms];
  ApproxTerm a[kFusedMaxTerms];
  int nterms;
  RefineRange r[kMaxBounds];
  int nranges;
  int zero_start;         // candidate mode: every bit starts at zero, so misses write nothing
  uint32_t *out;
  unsigned long long *count;
};

constexpr int kRefineRows = 2;  // rows per thread and iteration of refine_kernel

// Launched right behind the sieve (or the zero fill of a candidate plan)
// with programmatic stream serialization, so that its first blocks run
// beside that grid: every block resolves the ranges' ends itself (binary
// searches in the sorted values) and loads and tests its first rows, and
// waits for the bitmap only before its first atomic.
__global__ void __launch_bounds__(kThreads) refine_kernel(const __grid_constant__ RefineParams p) {
  __shared__ unsigned long long s_begin[kMaxBounds], s_end[kMaxBounds];
  __shared__ long long part[kThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < p.nranges; r += kThreads / 32) {
    const uint64_t a = resolve_end(p.r[r], p.r[r].e0);
    const uint64_t b = resolve_end(p.r[r], p.r[r].e1);
    if (lane == 0) {
      s_begin[r] = min(a, b);
      s_end[r] = max(a, b);
    }
  }
  __syncthreads();
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const long long delta = refine_rows<true, kRefineRows>(p.r, p.nranges, p.t, p.a, p.nterms, s_begin, s_end, tid,
                                                         stride, p.zero_start != 0, p.out);
  long long d = delta;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
  if (lane == 0) part[warp] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    wait_prerequisite();  // the count is the sieve's until then (also for a block without rows)
    long long s = 0;
    for (int i = 0; i < kThreads / 32; i++) s += part[i];
    if (s) atomicAdd(p.count, (unsigned long long)s);
  }
}

int blocks_for(uint64_t items, int sm_count, int per_sm) {
  uint64_t b = (items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)sm_count * per_sm;
  if (b > cap) b = cap;
  return (int)std::max<uint64_t>(1, b);
}

}  // namespace

GpuBinDex::~GpuBinDex() {
  if (sval) cudaFree(sval);
  if (spos) cudaFree(spos);
  if (fv) cudaFree(fv);
}

namespace {
template <class T>
T *dev_alloc(size_t count) {
  T *p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    throw Error(RTS_ERR_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  return p;
}
struct DevFree {
  void *p;
  ~DevFree() {
    if (p) cudaFree(p);
  }
};
}  // namespace

uint64_t count_fv_mismatches(const uint32_t *col, uint64_t n, const uint32_t *d_start, int K, const uint32_t *fv,
                             uint64_t fv_stride, unsigned long long *d_bad, int sm_count, cudaStream_t s) {
  RTS_CUDA(cudaMemsetAsync(d_bad, 0, 8, s));
  if (K > 1) launch_fv<true>(col, n, d_start, K, const_cast<uint32_t *>(fv), fv_stride, d_bad, sm_count, s);
  RTS_CUDA(cudaGetLastError());
  unsigned long long bad = 0;
  RTS_CUDA(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, s));
  RTS_CUDA(cudaStreamSynchronize(s));
  return bad;
}

std::unique_ptr<GpuBinDex> build_bindex(const uint32_t *col, uint64_t n, int K, int sm_count, cudaStream_t s) {
  if (K < 2 || K > 4096) throw Error(RTS_ERR_ARG, "K must be in [2, 4096]");
  if (n < (uint64_t)K) throw Error(RTS_ERR_ARG, "BinDex needs at least K rows");
  if (n >= (1ull << 32)) throw Error(RTS_ERR_ARG, "BinDex supports fewer than 2^32 rows per column");
  auto b = std::make_unique<GpuBinDex>();
  b->K = K;
  b->n = n;
  b->sval = dev_alloc<uint32_t>(n);
  b->spos = dev_alloc<uint32_t>(n);
  uint32_t *ids = dev_alloc<uint32_t>(n);
  DevFree f_ids{ids};
  iota_kernel<<<blocks_for(n, sm_count, 8), kThreads, 0, s>>>(ids, n);
  size_t temp_bytes = 0;
  RTS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, col, b->sval, ids, b->spos, (int64_t)n, 0, 32, s));
  void *temp = dev_alloc<char>(temp_bytes);
  DevFree f_temp{temp};
  RTS_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, col, b->sval, ids, b->spos, (int64_t)n, 0, 32, s));

  uint32_t *d_start = dev_alloc<uint32_t>(K);
  DevFree f_start{d_start};
  unsigned long long *d_rank = dev_alloc<unsigned long long>(K);
  DevFree f_rank{d_rank};
  area_kernel<<<(K * 32 + kThreads - 1) / kThreads, kThreads, 0, s>>>(b->sval, n, K, d_start, d_rank);
  const uint64_t m = (n + kSampleStride - 1) / kSampleStride;
  uint32_t *d_sample = dev_alloc<uint32_t>(m);
  DevFree f_sample{d_sample};
  sample_kernel<<<blocks_for(m, sm_count, 4), kThreads, 0, s>>>(b->sval, n, d_sample, m, kSampleStride);

  b->fv_stride = (((n + 31) >> 5) + 3) / 4 * 4;
  if (K > 1) {
    b->fv = dev_alloc<uint32_t>((size_t)(K - 1) * b->fv_stride);
    RTS_CUDA(cudaMemsetAsync(b->fv, 0, (size_t)(K - 1) * b->fv_stride * 4, s));
    launch_fv<false>(col, n, d_start, K, b->fv, b->fv_stride, nullptr, sm_count, s);
  }
  RTS_CUDA(cudaGetLastError());
  b->start.resize(K);
  std::vector<unsigned long long> rk(K);
  b->sample.resize(m);
  RTS_CUDA(cudaMemcpyAsync(b->start.data(), d_start, K * 4, cudaMemcpyDeviceToHost, s));
  RTS_CUDA(cudaMemcpyAsync(rk.data(), d_rank, K * 8, cudaMemcpyDeviceToHost, s));
  RTS_CUDA(cudaMemcpyAsync(b->sample.data(), d_sample, m * 4, cudaMemcpyDeviceToHost, s));
  uint32_t ends[2];
  RTS_CUDA(cudaMemcpyAsync(&ends[0], b->sval, 4, cudaMemcpyDeviceToHost, s));
  RTS_CUDA(cudaMemcpyAsync(&ends[1], b->sval + n - 1, 4, cudaMemcpyDeviceToHost, s));
  RTS_CUDA(cudaStreamSynchronize(s));
  b->first_rank.assign(rk.begin(), rk.end());
  b->min_val = ends[0];
  b->max_val = ends[1];
  return b;
}

namespace {

// Estimated lower_bound(sorted, b) from the host sample, and the exact
// search window [wlo, whi] that must contain it.
struct Est {
  uint64_t est, wlo, whi;
};
Est estimate(const GpuBinDex &B, uint32_t b) {
  const auto &s = B.sample;
  const uint64_t j = std::lower_bound(s.begin(), s.end(), b) - s.begin();
  Est e;
  e.wlo = j == 0 ? 0 : (j - 1) * kSampleStride + 1;
  e.whi = std::min<uint64_t>(B.n, j * kSampleStride);
  if (e.whi < e.wlo) e.whi = e.wlo;
  e.est = (e.wlo + e.whi) / 2;
  return e;
}

// Nearest approximation of "x < b": returns the filter-vector index (-1 =
// constant zero, K-1 = constant one) and its rank.
struct Approx {
  int k;
  uint64_t rank;
};
Approx nearest(const GpuBinDex &B, uint64_t est) {
  Approx best{-1, 0};
  uint64_t bd = est;  // distance to constant zero (rank 0)
  if (B.n - est < bd) {
    best = {B.K - 1, B.n};
    bd = B.n - est;
  }
  // fv[k] = (x < S[k+1]) has rank first_rank[k+1]
  const auto &fr = B.first_rank;
  auto it = std::lower_bound(fr.begin() + 1, fr.end(), est);
  for (int d = -1; d <= 0; d++) {
    auto jt = it + d;
    if (jt < fr.begin() + 1 || jt >= fr.end()) continue;
    const uint64_t r = *jt;
    const uint64_t dist = r > est ? r - est : est - r;
    if (dist < bd) {
      bd = dist;
      best = {(int)(jt - fr.begin()) - 1, r};
    }
  }
  return best;
}

}  // namespace

void bindex_query(rts_ctx *ctx, const rts_term *terms, int nterms, uint32_t *out, unsigned long long *count,
                  cudaStream_t s) {
  // Merge terms per column, drop always-true ones (as the fused planner).
  std::vector<int> cols;
  std::vector<uint32_t> lo, hi;
  bool empty = false;
  for (int i = 0; i < nterms; i++) {
    const rts_term &t = terms[i];
    if (t.column < 0 || t.column >= (int)ctx->cols.size()) throw Error(RTS_ERR_ARG, "term column out of range");
    if (t.lo > t.hi) empty = true;
    auto it = std::find(cols.begin(), cols.end(), (int)t.column);
    if (it == cols.end()) {
      cols.push_back(t.column);
      lo.push_back(t.lo);
      hi.push_back(t.hi);
    } else {
      size_t k = it - cols.begin();
      lo[k] = std::max(lo[k], t.lo);
      hi[k] = std::min(hi[k], t.hi);
      if (lo[k] > hi[k]) empty = true;
    }
  }
  const uint64_t n = ctx->nrows;
  int launches = 0;
  if (empty) {
    launch_fill_range(out, n, false, count, ctx->sm_count, s);
    ctx->launches += 2;
    return;
  }
  std::vector<int> tc;
  std::vector<uint32_t> tlo, thi;
  for (size_t k = 0; k < cols.size(); k++) {
    if (lo[k] == 0 && hi[k] == 0xFFFFFFFFu) continue;
    tc.push_back(cols[k]);
    tlo.push_back(lo[k]);
    thi.push_back(hi[k]);
  }
  const int T = (int)tc.size();
  if (T == 0) {
    launch_fill_range(out, n, true, count, ctx->sm_count, s);
    ctx->launches += 2;
    return;
  }
  if (T > kFusedMaxTerms) throw Error(RTS_ERR_ARG, "BinDex path takes at most 16 constrained columns per query");
  for (int c : tc)
    if (c >= (int)ctx->bindex.size() || !ctx->bindex[c])
      throw Error(RTS_ERR_STATE, "column " + std::to_string(c) + " has no BinDex (rts_build_bindex)");

  // Per term: bounds, estimates, nearest approximations.
  struct TermPlan {
    bool has_lo, has_hi;
    Est e_lo, e_hi;
    Approx a_lo, a_hi;
    uint64_t match_est, refine_est;
  };
  std::vector<TermPlan> tp(T);
  double sieve_cost = (double)n / 8;  // result write
  double per_row_refine = 8.0 + 32.0 * (T - 1) + 32.0;
  int best_cand = -1;
  double best_cand_cost = 1e300;
  for (int t = 0; t < T; t++) {
    const GpuBinDex &B = *ctx->bindex[tc[t]];
    TermPlan &p = tp[t];
    p.has_lo = tlo[t] > 0;
    p.has_hi = thi[t] < 0xFFFFFFFFu;
    uint64_t r_lo = 0, r_hi = n;
    p.refine_est = 0;
    if (p.has_lo) {
      p.e_lo = estimate(B, tlo[t]);
      p.a_lo = nearest(B, p.e_lo.est);
      r_lo = p.e_lo.est;
      p.refine_est += p.a_lo.rank > r_lo ? p.a_lo.rank - r_lo : r_lo - p.a_lo.rank;
      if (p.a_lo.k >= 0 && p.a_lo.k < B.K - 1) sieve_cost += (double)n / 8;
    }
    if (p.has_hi) {
      p.e_hi = estimate(B, thi[t] + 1);
      p.a_hi = nearest(B, p.e_hi.est);
      r_hi = p.e_hi.est;
      p.refine_est += p.a_hi.rank > r_hi ? p.a_hi.rank - r_hi : r_hi - p.a_hi.rank;
      if (p.a_hi.k >= 0 && p.a_hi.k < B.K - 1) sieve_cost += (double)n / 8;
    }
    p.match_est = r_hi > r_lo ? r_hi - r_lo : 0;
    sieve_cost += (double)p.refine_est * per_row_refine;
    const double cand = (double)n / 8 + (double)(p.match_est + 2 * kSampleStride) * per_row_refine;
    if (cand < best_cand_cost) {
      best_cand_cost = cand;
      best_cand = t;
    }
  }

  RefineParams rp;
  memset(&rp, 0, sizeof rp);
  rp.nterms = T;
  for (int t = 0; t < T; t++) rp.t[t] = {ctx->cols[tc[t]], tlo[t], thi[t] - tlo[t]};
  rp.out = out;
  rp.count = count;
  auto end_of = [&](const Est &e, uint32_t b) {
    RangeEnd r;
    memset(&r, 0, sizeof r);
    r.kind = 1;
    r.b = b;
    r.wlo = e.wlo;
    r.whi = e.whi;
    return r;
  };
  auto end_rank = [&](uint64_t rank) {
    RangeEnd r;
    memset(&r, 0, sizeof r);
    r.kind = 0;
    r.rank = rank;
    return r;
  };

  SieveParams sp;
  memset(&sp, 0, sizeof sp);
  sp.out = out;
  sp.count = count;
  sp.words = words_for(n);
  const uint32_t rem = (uint32_t)(n & 31);
  sp.tail_mask = rem ? ~(0xFFFFFFFFu >> rem) : 0xFFFFFFFFu;
  sp.vec = ((uintptr_t)out & 15) == 0;
  // The value an approximation stands for: fv[k] holds x < start[k+1];
  // k = -1 is no row (x < 0), k = K-1 every row (x < 2^32).
  auto approx_value = [&](const GpuBinDex &B, const Approx &a) -> uint64_t {
    return a.k < 0 ? 0 : a.k >= B.K - 1 ? (1ull << 32) : B.start[a.k + 1];
  };
  // A range's rows are those whose value lies between its ends' bounds.
  auto window = [](RefineRange &rg, uint64_t v0, uint64_t v1) {
    const uint64_t a = std::min(v0, v1), b = std::max(v0, v1);
    rg.wok = a < b;
    rg.wlo = (uint32_t)a;
    rg.wspan = a < b ? (uint32_t)(b - 1 - a) : 0u;
  };
  if (best_cand_cost < sieve_cost) {
    // Candidate mode: start from zero, re-test the matches of one term.
    const int t = best_cand;
    const GpuBinDex &B = *ctx->bindex[tc[t]];
    RefineRange &rg = rp.r[0];
    rg.sval = B.sval;
    rg.spos = B.spos;
    rg.term = t;
    rg.e0 = tp[t].has_lo ? end_of(tp[t].e_lo, tlo[t]) : end_rank(0);
    rg.e1 = tp[t].has_hi ? end_of(tp[t].e_hi, thi[t] + 1) : end_rank(n);
    window(rg, tp[t].has_lo ? tlo[t] : 0, tp[t].has_hi ? (uint64_t)thi[t] + 1 : (1ull << 32));
    rp.nranges = 1;
    rp.zero_start = 1;
  } else {
    sp.nterms = T;
    for (int t = 0; t < T; t++) {
      const GpuBinDex &B = *ctx->bindex[tc[t]];
      SieveTerm &st = sp.t[t];
      // upper: x < hi+1 ; lower: x < lo (negated in the sieve)
      if (!tp[t].has_hi || tp[t].a_hi.k == B.K - 1) { st.U = nullptr; st.u_const = ~0u; }
      else if (tp[t].a_hi.k < 0) { st.U = nullptr; st.u_const = 0u; }
      else st.U = B.fv + (uint64_t)tp[t].a_hi.k * B.fv_stride;
      if (!tp[t].has_lo || tp[t].a_lo.k < 0) { st.L = nullptr; st.l_const = 0u; }
      else if (tp[t].a_lo.k == B.K - 1) { st.L = nullptr; st.l_const = ~0u; }
      else st.L = B.fv + (uint64_t)tp[t].a_lo.k * B.fv_stride;
      // the same verdict as a value range: lb <= x < ub
      const uint64_t ub = tp[t].has_hi ? approx_value(B, tp[t].a_hi) : (1ull << 32);
      const uint64_t lb = tp[t].has_lo ? approx_value(B, tp[t].a_lo) : 0;
      rp.a[t].ok = lb < ub;
      rp.a[t].lo = (uint32_t)lb;
      rp.a[t].span = lb < ub ? (uint32_t)(ub - 1 - lb) : 0u;
      if (tp[t].has_hi) {
        RefineRange &rg = rp.r[rp.nranges++];
        rg.sval = B.sval;
        rg.spos = B.spos;
        rg.term = t;
        rg.e0 = end_of(tp[t].e_hi, thi[t] + 1);
        rg.e1 = end_rank(tp[t].a_hi.rank);
        window(rg, (uint64_t)thi[t] + 1, approx_value(B, tp[t].a_hi));
      }
      if (tp[t].has_lo) {
        RefineRange &rg = rp.r[rp.nranges++];
        rg.sval = B.sval;
        rg.spos = B.spos;
        rg.term = t;
        rg.e0 = end_of(tp[t].e_lo, tlo[t]);
        rg.e1 = end_rank(tp[t].a_lo.rank);
        window(rg, tlo[t], approx_value(B, tp[t].a_lo));
      }
    }
  }
  if (!ctx->query_slots) {
    if (cudaMalloc(&ctx->query_slots, kQuerySlots * sizeof(QuerySlot)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "device allocation failed");
    }
    RTS_CUDA(cudaMemsetAsync(ctx->query_slots, 0, kQuerySlots * sizeof(QuerySlot), s));
  }
  QuerySlot *slot = ctx->query_slots + (ctx->query_next++ % kQuerySlots);
  sp.slot = slot;
  sp.nranges = rp.nranges;
  for (int r = 0; r < rp.nranges; r++) sp.r[r] = rp.r[r];
  uint64_t est_rows = 0;
  for (int t = 0; t < T; t++) est_rows += tp[t].refine_est;
  if (rp.zero_start) est_rows = tp[best_cand].match_est;
  // A refine set estimated at a few rows (exact ends can differ from the
  // estimates by a sample stride) costs the sieve's last block less than a
  // launch of its own.
  if (est_rows <= kRefineInSieveRows) {
    sp.refine_here = 1;
    sp.zero_start = rp.zero_start;
    sp.rnterms = rp.nterms;
    for (int t = 0; t < rp.nterms; t++) {
      sp.rt[t] = rp.t[t];
      sp.ra[t] = rp.a[t];
    }
  }
  const uint64_t nvec = sp.words / 4 + 1;
  sieve_kernel<<<blocks_for(nvec, ctx->sm_count, 4), kThreads, 0, s>>>(sp);  // one wave: 48 registers allow 5 blocks per SM
  launches++;
  if (rp.nranges && !sp.refine_here) {
    cudaLaunchConfig_t cfg = {};
    const uint64_t threads = (std::max<uint64_t>(est_rows, 1) + kRefineRows - 1) / kRefineRows;
    cfg.gridDim = dim3(blocks_for(threads, ctx->sm_count, 8));
    cfg.blockDim = dim3(kThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    RTS_CUDA(cudaLaunchKernelEx(&cfg, refine_kernel, rp));
    launches++;
  }
  RTS_CUDA(cudaGetLastError());
  ctx->launches += launches;
}

}  // namespace rts

extern "C" {

rts_status rts_build_bindex(rts_ctx *ctx, int32_t column, int32_t K) {
  rts::Range nvtx_range_("rts_build_bindex");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (ctx->cols.empty()) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (column < 0 || column >= (int)ctx->cols.size()) throw rts::Error(RTS_ERR_ARG, "column out of range");
    rts::DeviceGuard device_guard(ctx->device);
    if (ctx->bindex.size() < ctx->cols.size()) ctx->bindex.resize(ctx->cols.size());
    ctx->bindex[column].reset();
    auto b = rts::build_bindex(ctx->cols[column], ctx->nrows, K, ctx->sm_count, nullptr);
    ctx->launches += 5;
    ctx->bindex[column] = std::move(b);
    return RTS_OK;
  } catch (const rts::Error &e) {
    ctx->err = e.what();
    return rts::set_thread_error(e.code, e.what());
  } catch (const std::exception &e) {
    ctx->err = e.what();
    return rts::set_thread_error(RTS_ERR_NOMEM, e.what());
  }
}

rts_status rts_drop_bindex(rts_ctx *ctx, int32_t column) {
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  if (column < 0 || column >= (int)ctx->bindex.size()) {
    ctx->err = "column out of range";
    return rts::set_thread_error(RTS_ERR_ARG, ctx->err);
  }
  ctx->bindex[column].reset();
  return RTS_OK;
}

rts_status rts_bindex_areas(const rts_ctx *ctx, int32_t column, uint32_t *starts, uint64_t *first_rank, int32_t K) {
  if (!ctx || column < 0 || column >= (int)ctx->bindex.size() || !ctx->bindex[column])
    return rts::set_thread_error(RTS_ERR_STATE, "column has no BinDex");
  const rts::GpuBinDex &B = *ctx->bindex[column];
  if (K != B.K) return rts::set_thread_error(RTS_ERR_ARG, "K differs from the index's K");
  for (int k = 0; k < K; k++) {
    if (starts) starts[k] = B.start[k];
    if (first_rank) first_rank[k] = B.first_rank[k];
  }
  return RTS_OK;
}

rts_status rts_bindex_filter_vector(rts_ctx *ctx, int32_t column, int32_t k, uint32_t *host_out) {
  if (!ctx || column < 0 || column >= (int)ctx->bindex.size() || !ctx->bindex[column])
    return rts::set_thread_error(RTS_ERR_STATE, "column has no BinDex");
  const rts::GpuBinDex &B = *ctx->bindex[column];
  if (k < 0 || k >= B.K - 1 || !host_out) return rts::set_thread_error(RTS_ERR_ARG, "bad filter vector index");
  try {
    rts::DeviceGuard device_guard(ctx->device);
    RTS_CUDA(cudaMemcpy(host_out, B.fv + (uint64_t)k * B.fv_stride, rts::words_for(B.n) * 4,
                        cudaMemcpyDeviceToHost));
    return RTS_OK;
  } catch (const std::exception &e) {
    return rts::set_thread_error(rts::status_of(e), e.what());
  }
}

rts_status rts_bindex_scan_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap,
                                 uint64_t *dev_count, void *stream) {
  rts::Range nvtx_range_("rts_bindex_scan_async");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (ctx->cols.empty()) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (!dev_bitmap || !dev_count) throw rts::Error(RTS_ERR_ARG, "null result pointer");
    if (nterms < 0 || (nterms > 0 && !terms)) throw rts::Error(RTS_ERR_ARG, "bad term list");
    rts::DeviceGuard device_guard(ctx->device);
    rts::bindex_query(ctx, terms, nterms, dev_bitmap, reinterpret_cast<unsigned long long *>(dev_count),
                      (cudaStream_t)stream);
    return RTS_OK;
  } catch (const std::exception &e) {
    ctx->err = e.what();
    return rts::set_thread_error(rts::status_of(e), e.what());
  }
}


}  // extern "C"
