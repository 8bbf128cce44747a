// Batched scan: many queries in one pass over the columns.
//
// The reference answers one query per loop iteration and re-reads its
// columns every time (bindex_cuda.cpp:1827-1986).  Here a batch is split
// into passes of up to 512 queries over up to 8 constrained columns, and
// each pass is one persistent kernel that streams every column chunk from
// HBM once and evaluates all the pass's queries on it:
//
//   * Per pass and column, the host collects the query bounds on that
//     column (lo and hi+1 of every term) into a sorted boundary list B.  The
//     boundaries cut the value domain into intervals, and every query's
//     verdict on the column is constant over an interval.  The kernel finds a
//     row's interval ("position", #boundaries <= x) with a bucket index
//     (linear or log-linear buckets, whichever spreads this column's
//     boundaries better) plus a short search, all in shared memory.
//   * A mask table gives, per position, one bit per query slot (G words of
//     32 slots).  A row's verdict for all queries is the AND of its columns'
//     table rows: C shared-memory loads per row and group of 32 queries
//     instead of up to 2*C compares per row and query.
//   * Variant 4 (default, batch4.cuh): CTA-wide blocks of 512-4096 rows;
//     each lane ANDs the masks of 32 rows for one group, transposes the
//     32x32 bit block in registers and stages the words for whole-line
//     stores.  Passes of at most 20 queries skip the tables and test each
//     term directly (batch_few.cuh).  Variant 3 (below): 256-query passes
//     with one 256-row block per warp, kept as an autotuner candidate.
//   * Counts are kept per lane in registers and flushed once per CTA.
// Queries with an empty term, with no constrained column, or with more than
// eight constrained columns are answered outside these kernels (fill or
// fused scan), so the result of every query equals the single-query path.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "batch_plan.h"
#include "rts_internal.h"

namespace rts {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kSlots = 256;         // queries per pass
constexpr int kGroups = kSlots / 32;
constexpr int kMaxCols = 8;         // constrained columns per pass
constexpr int kTilesPerBlock = 8;   // 8 tiles x 32 rows = one 32-byte sector per query
constexpr int kStageWords = kSlots * kTilesPerBlock;  // per warp
template <int CMAX>
constexpr int kPosWords = 36 * CMAX;  // per warp: 32 rows + one padding row per 8

struct BatchPass {
  const uint32_t *col[kMaxCols];
  uint32_t m[kMaxCols];         // boundaries of column c
  uint32_t bmin[kMaxCols];      // B[0]
  uint32_t bmax[kMaxCols];      // B[m-1]
  uint32_t shift[kMaxCols];     // linear buckets: bucket = (x - bmin) >> shift
  uint32_t lgm[kMaxCols];       // > 0: log-linear buckets with lgm mantissa bits (bucket_of)
  uint32_t tab_off[kMaxCols];   // word offsets into the pass blob
  uint32_t bnd_off[kMaxCols];
  uint32_t bkt_off[kMaxCols];   // uint16 bucket starts, nbk+1 entries
  uint32_t nbk[kMaxCols];       // buckets of column c
  int ncols;
  uint32_t blob_words;          // words of the blob copied to shared memory
  const uint32_t *blob;         // tables | boundaries | buckets | slot map (global)
  uint32_t slot_off;            // word offset of the 256-entry slot -> query map
  uint32_t *out;
  uint64_t stride_words;
  unsigned long long *counts;
  uint64_t nrows;
  uint64_t words;               // bitmap words of one query
  uint64_t block_begin;         // first block of the range (256 rows, 1024 for variant 4)
  uint64_t nblocks;             // end of the range, in blocks
  int vec_store;                // bitmaps 16-byte aligned (out and stride)
  uint32_t word_bytes;          // 4, passed at run time (see the mask loop of batch4_kernel)
  const uint2 *pre;             // shared positions: the pass's table word offsets of row r at pre[r - pre_row0]
  uint64_t pre_row0;
};

// Log-linear bucket of v >= 0 with M mantissa bits: v itself below 2^M,
// else 2^M buckets per octave, (e - M + 1) * 2^M + the M bits under the
// leading one for v in [2^e, 2^(e+1)).  Monotone in v; at most
// (33 - M) * 2^M buckets.  Skewed columns (a few dense small values and a
// long tail) spread their boundaries over these buckets far more evenly
// than over linear ones.
__host__ __device__ __forceinline__ uint32_t bucket_of(uint32_t v, uint32_t M) {
#ifdef __CUDA_ARCH__
  const int e = 31 - __clz(v);  // -1 for v = 0
#else
  const int e = v ? 31 - __builtin_clz(v) : -1;
#endif
  const uint32_t sh = e > (int)M ? (uint32_t)(e - (int)M) : 0u;
  return (sh << M) + (v >> sh);
}

// Position of x among the boundaries of column c from the bucket index
// alone, without a loop: exact (and *exact set) when x's bucket holds at
// most two boundaries, the usual case; callers redo the others with
// position().  Every load stays inside the pass blob: a value below B[0]
// or above the last bucket is clamped to a bucket, and B[lo + 1] past the
// boundaries reads the bucket index that follows them.
__device__ __forceinline__ uint32_t position_fast(const BatchPass &p, const uint32_t *sm, int c, uint32_t x,
                                                  bool &exact) {
  const uint32_t v = x - p.bmin[c];
  const uint32_t k = min(p.lgm[c] ? bucket_of(v, p.lgm[c]) : v >> p.shift[c], p.nbk[c] - 1);
  const uint16_t *bk = reinterpret_cast<const uint16_t *>(sm + p.bkt_off[c]);
  const uint32_t lo = bk[k], hi = bk[k + 1];
  const uint32_t *B = sm + p.bnd_off[c];
  const uint32_t b0 = B[lo], b1 = B[lo + 1];
  const bool below = x < p.bmin[c];
  exact = below || hi - lo <= 2;
  const uint32_t pos = lo + (hi > lo && b0 <= x) + (hi > lo + 1 && b1 <= x);
  return below ? 0u : pos;
}

// Position of x among the boundaries of column c: #{B[i] <= x}.
__device__ __forceinline__ uint32_t position(const BatchPass &p, const uint32_t *sm, int c, uint32_t x) {
  const uint32_t m = p.m[c];
  if (m == 0 || x < p.bmin[c]) return 0;
  if (x >= p.bmax[c]) return m;
  const uint32_t v = x - p.bmin[c];
  const uint32_t k = p.lgm[c] ? bucket_of(v, p.lgm[c]) : v >> p.shift[c];
  const uint16_t *bk = reinterpret_cast<const uint16_t *>(sm + p.bkt_off[c]);
  uint32_t lo = bk[k], hi = bk[k + 1];  // boundaries of bucket k: B[lo..hi)
  const uint32_t *B = sm + p.bnd_off[c];
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (B[mid] <= x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Shared positions.  A batch of several table passes over the same columns
// searches every row's position once per column, among the union of the
// passes' boundaries (each pass's boundaries are a subset of the union, so
// a union position fixes the position in every pass), and reads all the
// passes' table word offsets for it from one entry of a per-column map.
// The passes then read four 16-bit offsets per row instead of searching
// (batch4_kernel with PRE).  Pass column c is union column c.
constexpr int kMaxPrePasses = kMaxSharedPasses;
constexpr uint32_t kPreMaxBuckets = 4096;  // per union column

// A union column: its m sorted distinct boundaries B, their bucket index and
// the map.  A value x is clamped to `origin` (B[0] - 1, or 0) and taken
// relative to it, v = max(x, origin) - origin; its bucket is
// k = ((s - L) << M) + (v >> s) with s = max(floor(log2 v) - M, L)
// (floor(log2 0) = -1): buckets of 2^L values below 2^(M+L+1), then 2^M
// buckets per octave (M = 31: linear buckets only), clamped to nbk - 1.
// Bucket entry k is base | n << 16: base = #{B <= the bucket's first value},
// n = #{B in the bucket above its first value} (in the last bucket: every
// boundary above it), so that pos(x) = base + #{B[base, base + n) <= x},
// and n = 0 in most buckets.  The map entry of union position p holds the
// passes' table word offsets for it, two per word (pass 2w in the low half
// of word w): (npass + 1) / 2 words.
struct PreCol {
  const uint32_t *col;
  uint32_t origin, M, L, nbk, m;
  uint32_t bkt_off, bnd_off, map_off;  // word offsets into the union blob
};

struct PreParams {
  PreCol c[4];
  int ncols;                   // the passes' columns
  int npass;                   // 1..kMaxPrePasses
  const uint32_t *blob;        // union blob (global): per column buckets | boundaries | map
  uint32_t blob_words;
  uint64_t row_begin, row_end;
  uint2 *out;                  // out[q * stride + (row - row_begin)]: pass q's four offsets, two per word
  uint64_t stride;             // pre_stride(row_end - row_begin)
  int vec;                     // every column 8-byte aligned at row_begin
};

__host__ __device__ __forceinline__ uint32_t pre_bucket(const PreCol &pc, uint32_t x) {
  const uint32_t v = (x > pc.origin ? x : pc.origin) - pc.origin;
#ifdef __CUDA_ARCH__
  const int e = 31 - __clz(v);  // -1 for v = 0
#else
  const int e = v ? 31 - __builtin_clz(v) : -1;
#endif
  const int s = e - (int)pc.M > (int)pc.L ? e - (int)pc.M : (int)pc.L;
  const uint32_t k = (((uint32_t)s - pc.L) << pc.M) + (v >> s);
  return k < pc.nbk - 1 ? k : pc.nbk - 1;
}

// Union position of x in column pc: #{B <= x}.
__host__ __device__ __forceinline__ uint32_t pre_position(const PreCol &pc, const uint32_t *blob, uint32_t x) {
  const uint32_t w = blob[pc.bkt_off + pre_bucket(pc, x)];
  uint32_t pos = w & 0xFFFFu, n = w >> 16;
  const uint32_t *B = blob + pc.bnd_off;
  while (n) {  // lower bound among B[pos, pos + n)
    const uint32_t h = n >> 1;
    if (B[pos + h] <= x) {
      pos += h + 1;
      n -= h + 1;
    } else {
      n = h;
    }
  }
  return pos;
}

constexpr int kPreThreads = 1024;  // two-pass batches: two blocks per SM, 64 warps over two table copies
constexpr int kPrePairs = 2;  // row pairs per thread and iteration: their loads and searches overlap
constexpr uint64_t kPreTile = (uint64_t)kPreThreads * kPrePairs * 2;  // rows of one block iteration

// Rows of a pass's slice of the scratch: even, so that every pass's slice
// starts 16-byte aligned and a row pair is one 16-byte store.
__host__ __device__ __forceinline__ uint64_t pre_stride(uint64_t rows) { return (rows + 1) & ~1ull; }

// U: union columns; NW: map words per entry, 1 for two passes, 2 for three
// or four.  A thread takes row pairs; tiles wholly inside the range with
// 8-byte aligned columns (P.vec) load each column's pair as one uint2 and
// store each pass's pair as one uint4, without per-row checks.
template <int U, int NW>
__global__ void __launch_bounds__(kPreThreads, NW == 1 ? 2 : 1) pre_kernel(const __grid_constant__ PreParams P) {
  extern __shared__ __align__(16) uint32_t smem[];
  for (uint32_t i = threadIdx.x; i < P.blob_words; i += blockDim.x) smem[i] = __ldg(P.blob + i);
  __syncthreads();
  for (uint64_t base = P.row_begin + (uint64_t)blockIdx.x * kPreTile; base < P.row_end;
       base += (uint64_t)gridDim.x * kPreTile) {
    const bool full = P.vec && base + kPreTile <= P.row_end;
    uint32_t x[kPrePairs][2][U];
#pragma unroll
    for (int j = 0; j < kPrePairs; j++) {
      const uint64_t row = base + 2 * (threadIdx.x + (uint64_t)j * kPreThreads);
#pragma unroll
      for (int c = 0; c < U; c++) {
        if (full) {
          const uint2 v = __ldg(reinterpret_cast<const uint2 *>(P.c[c].col + row));
          x[j][0][c] = v.x;
          x[j][1][c] = v.y;
        } else {
          x[j][0][c] = row < P.row_end ? __ldg(P.c[c].col + row) : 0u;
          x[j][1][c] = row + 1 < P.row_end ? __ldg(P.c[c].col + row + 1) : 0u;
        }
      }
    }
    // map entries of every row and column; the searches of the thread's rows
    // and columns are independent, so their shared-memory loads overlap
    uint32_t e[kPrePairs][2][4][NW];
#pragma unroll
    for (int j = 0; j < kPrePairs; j++)
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if (c < U) {
            const uint32_t *ent = smem + P.c[c].map_off + pre_position(P.c[c], smem, x[j][h][c]) * NW;
            if (NW == 2) {
              const uint2 w = *reinterpret_cast<const uint2 *>(ent);
              e[j][h][c][0] = w.x;
              e[j][h][c][NW - 1] = w.y;
            } else {
              e[j][h][c][0] = *ent;
            }
          } else {
#pragma unroll
            for (int w = 0; w < NW; w++) e[j][h][c][w] = 0u;
          }
        }
#pragma unroll
    for (int j = 0; j < kPrePairs; j++) {
      const uint64_t row = base + 2 * (threadIdx.x + (uint64_t)j * kPreThreads);
#pragma unroll
      for (int q = 0; q < 2 * NW; q++) {
        if (q >= P.npass) break;
        const int w = q >> 1;
        const uint32_t sel = (q & 1) ? 0x7632u : 0x5410u;  // the pass's halves of two entries
        uint2 o[2];
#pragma unroll
        for (int h = 0; h < 2; h++)
          o[h] = make_uint2(__byte_perm(e[j][h][0][w], e[j][h][1][w], sel),
                            __byte_perm(e[j][h][2][w], e[j][h][3][w], sel));
        uint2 *dst = P.out + q * P.stride + (row - P.row_begin);
        if (full) {
          *reinterpret_cast<uint4 *>(dst) = make_uint4(o[0].x, o[0].y, o[1].x, o[1].y);
        } else {
          if (row < P.row_end) dst[0] = o[0];
          if (row + 1 < P.row_end) dst[1] = o[1];
        }
      }
    }
  }
}

// 8x8 bit transposes in each byte lane of eight registers: on return, bit r
// of byte b of x[c] is bit c of byte b of the input x[r].
__device__ __forceinline__ void transpose8x8x4(uint32_t (&x)[8]) {
#pragma unroll
  for (int r = 0; r < 4; r++) {
    uint32_t t = ((x[r] >> 4) ^ x[r + 4]) & 0x0F0F0F0Fu;
    x[r + 4] ^= t;
    x[r] ^= t << 4;
  }
#pragma unroll
  for (int base = 0; base < 8; base += 4) {
#pragma unroll
    for (int r = base; r < base + 2; r++) {
      uint32_t t = ((x[r] >> 2) ^ x[r + 2]) & 0x33333333u;
      x[r + 2] ^= t;
      x[r] ^= t << 2;
    }
  }
#pragma unroll
  for (int r = 0; r < 8; r += 2) {
    uint32_t t = ((x[r] >> 1) ^ x[r + 1]) & 0x55555555u;
    x[r + 1] ^= t;
    x[r] ^= t << 1;
  }
}

// Staging layout per warp: slot q, tile t -> row = q/4 holds the 32 words of
// slots 4*row..4*row+3 (8 tiles each) rotated by (row>>1)&31, so that both
// the per-tile writes (32 lanes, 32 different slots) and the per-sector
// reads (4 slots x 8 tiles) hit 32 different banks.
__device__ __forceinline__ uint32_t stage_index(uint32_t slot, uint32_t t) {
  const uint32_t row = slot >> 2;
  const uint32_t col = ((slot & 3) * 8 + t + ((row >> 1) & 31)) & 31;
  return row * 32 + col;
}

// Variant 3: 256-slot passes (8 groups), one 256-row block per warp.  Lane
// (s, g) owns rows s*8..s*8+7 of a 32-row tile for query group g; its eight
// 32-bit masks are bit-transposed in registers (three delta-swap stages)
// into bytes, the four lanes of a group exchange bytes so that each
// finalizes 8 queries' 32-row words, and the words are staged in shared
// memory until eight tiles make a full 32-byte sector per query, which the
// warp then stores with coalesced writes.
// CMAX: columns a pass may constrain (4 or 8); W: warps per CTA (8 or 16).
template <int CMAX, int W>
__global__ void __launch_bounds__(W * 32, 16 / W) batch_kernel(const __grid_constant__ BatchPass p) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *blob = smem;
  uint32_t *stage_all = smem + ((p.blob_words + 3) & ~3u);
  // positions of a warp's 32-row tile: row r at r*CMAX + (r/8)*CMAX words,
  // so the four rows read together (s*8+i, s = 0..3) sit in different banks
  uint32_t *posbuf_all = stage_all + W * kStageWords;
  unsigned int *cta_count = posbuf_all + W * kPosWords<CMAX>;

  for (uint32_t i = threadIdx.x; i < p.blob_words; i += blockDim.x) blob[i] = __ldg(p.blob + i);
  for (int i = threadIdx.x; i < kSlots; i += blockDim.x) cta_count[i] = 0;
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = lane >> 3, g = lane & 7;
  uint32_t *stage = stage_all + warp * kStageWords;
  uint32_t *posbuf = posbuf_all + warp * kPosWords<CMAX>;
  const int32_t *slot_query = reinterpret_cast<const int32_t *>(blob + p.slot_off);
  const int C = p.ncols;
  uint32_t tab_base[CMAX];  // this lane's word of table row 0, per column
#pragma unroll
  for (int c = 0; c < CMAX; c++) tab_base[c] = c < C ? p.tab_off[c] + g : 0u;
  const bool vec_store = p.vec_store;
  uint32_t cnt[8];
#pragma unroll
  for (int k = 0; k < 8; k++) cnt[k] = 0;

  const uint64_t gwarp = (uint64_t)blockIdx.x * W + warp;
  const uint64_t nwarps = (uint64_t)gridDim.x * W;
  for (uint64_t blk = p.block_begin + gwarp; blk < p.nblocks; blk += nwarps) {
    const uint64_t row0 = blk * (32 * kTilesPerBlock);
    // every column value of the block, loaded up front (lane = row in tile)
    uint32_t v[kTilesPerBlock][CMAX];
#pragma unroll
    for (int t = 0; t < kTilesPerBlock; t++) {
      const uint64_t row = row0 + 32 * t + lane;
#pragma unroll
      for (int c = 0; c < CMAX; c++)
        v[t][c] = (c < C && row < p.nrows) ? __ldg(p.col[c] + row) : 0u;
    }
#pragma unroll
    for (int t = 0; t < kTilesPerBlock; t++) {
      const uint64_t tile_row0 = row0 + 32 * t;
      // positions of this lane's row, one per column
      {
        uint32_t pv[CMAX];
#pragma unroll
        for (int c = 0; c < CMAX; c++) pv[c] = c < C ? position(p, blob, c, v[t][c]) : 0u;
        uint32_t *dst = posbuf + lane * CMAX + (lane >> 3) * CMAX;
#pragma unroll
        for (int c = 0; c < CMAX; c += 4)
          *reinterpret_cast<uint4 *>(dst + c) = make_uint4(pv[c], pv[c + 1], pv[c + 2], pv[c + 3]);
      }
      __syncwarp();
      // masks of rows s*8+i for group g
      uint32_t mk[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const uint32_t *pr = posbuf + (s * 8 + i) * CMAX + s * CMAX;
        uint32_t pos[CMAX];
#pragma unroll
        for (int c = 0; c < CMAX; c += 4) {
          const uint4 q4 = *reinterpret_cast<const uint4 *>(pr + c);
          pos[c] = q4.x;
          pos[c + 1] = q4.y;
          pos[c + 2] = q4.z;
          pos[c + 3] = q4.w;
        }
        uint32_t a = 0xFFFFFFFFu;
#pragma unroll
        for (int c = 0; c < CMAX; c++)
          if (c < C) a &= blob[tab_base[c] + pos[c] * kGroups];
        mk[7 - i] = a;  // reversed: bit r of the transposed byte is row 7-r
      }
      __syncwarp();
      transpose8x8x4(mk);
      // mk[c] byte b = 8 row bits (MSB = row s*8) of query 8b+c of group g.
      // Lane s finalizes byte lane b = s: in round d it sends byte lane s^d
      // of mk[0..3] and mk[4..7] (packed by byte permutes) to lane s^d of
      // its group and receives byte lane s from that lane.  The bytes from
      // round d belong at byte 3-d of V (static positions); the final word
      // wants source lane s^d's rows at byte 3-(s^d), i.e. output byte p
      // takes V's byte p^s.
      uint32_t rlo[4], rhi[4];
#pragma unroll
      for (int d = 0; d < 4; d++) {
        const uint32_t dst = (uint32_t)(s ^ d);
        const uint32_t sel = dst | ((dst + 4) << 4);
        const uint32_t lo4 = __byte_perm(__byte_perm(mk[0], mk[1], sel), __byte_perm(mk[2], mk[3], sel), 0x5410);
        const uint32_t hi4 = __byte_perm(__byte_perm(mk[4], mk[5], sel), __byte_perm(mk[6], mk[7], sel), 0x5410);
        rlo[d] = d == 0 ? lo4 : __shfl_xor_sync(kFull, lo4, 8 * d);
        rhi[d] = d == 0 ? hi4 : __shfl_xor_sync(kFull, hi4, 8 * d);
      }
      const uint32_t fix = (uint32_t)(0 ^ s) | ((uint32_t)(1 ^ s) << 4) | ((uint32_t)(2 ^ s) << 8) |
                           ((uint32_t)(3 ^ s) << 12);
      uint32_t w[8];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        // V byte 3-d = byte k of r[d]
        const uint32_t selk = (uint32_t)k | ((uint32_t)(k + 4) << 4);
        const uint32_t a = __byte_perm(rlo[3], rlo[2], selk);  // byte0 = r3.k, byte1 = r2.k
        const uint32_t b = __byte_perm(rlo[1], rlo[0], selk);  // byte0 = r1.k, byte1 = r0.k
        w[k] = __byte_perm(__byte_perm(a, b, 0x5410), 0, fix);
        const uint32_t c2 = __byte_perm(rhi[3], rhi[2], selk);
        const uint32_t d2 = __byte_perm(rhi[1], rhi[0], selk);
        w[k + 4] = __byte_perm(__byte_perm(c2, d2, 0x5410), 0, fix);
      }
      // w[k] is the word of query slot 32g + 8s + k for rows tile_row0..+31
      if (tile_row0 + 32 > p.nrows) {
        const uint64_t valid = tile_row0 < p.nrows ? p.nrows - tile_row0 : 0;
        const uint32_t vm = valid >= 32 ? 0xFFFFFFFFu : (valid ? ~(0xFFFFFFFFu >> valid) : 0u);
#pragma unroll
        for (int k = 0; k < 8; k++) w[k] &= vm;
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        cnt[k] += __popc(w[k]);
        stage[stage_index(32 * g + 8 * s + k, t)] = w[k];
      }
    }
    __syncwarp();
    // store: each lane writes one query's 8 words of this block (a full
    // 32-byte sector) with two 16-byte stores when the bitmaps are aligned
    const uint64_t word0 = blk * kTilesPerBlock;
    const bool full = word0 + kTilesPerBlock <= p.words;
#pragma unroll 2
    for (int j = 0; j < kSlots / 32; j++) {
      const uint32_t slot = 32 * j + lane;
      const int32_t q = slot_query[slot];
      uint32_t wv[kTilesPerBlock];
#pragma unroll
      for (int t = 0; t < kTilesPerBlock; t++) wv[t] = stage[stage_index(slot, t)];
      if (q >= 0) {
        uint32_t *dst = p.out + (uint64_t)q * p.stride_words + word0;
        if (vec_store && full) {
          reinterpret_cast<uint4 *>(dst)[0] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
          reinterpret_cast<uint4 *>(dst)[1] = make_uint4(wv[4], wv[5], wv[6], wv[7]);
        } else {
#pragma unroll
          for (int t = 0; t < kTilesPerBlock; t++)
            if (word0 + t < p.words) dst[t] = wv[t];
        }
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int k = 0; k < 8; k++)
    if (cnt[k]) atomicAdd(&cta_count[32 * g + 8 * s + k], cnt[k]);
  __syncthreads();
  for (int i = threadIdx.x; i < kSlots; i += blockDim.x) {
    const int32_t q = slot_query[i];
    if (q >= 0 && cta_count[i]) atomicAdd(p.counts + q, (unsigned long long)cta_count[i]);
  }
}

template <int CMAX, int W>
size_t smem_bytes(uint32_t blob_words) {
  return ((blob_words + 3) & ~3u) * 4 + (size_t)W * kStageWords * 4 + (size_t)W * kPosWords<CMAX> * 4 + kSlots * 4;
}

template <int CMAX, int W>
int blocks_per_sm(size_t smem) {
  static std::atomic<uint64_t> raised{0};
  raise_smem_limit(batch_kernel<CMAX, W>, raised, 227 * 1024);
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel<CMAX, W>, W * 32, smem) != cudaSuccess ||
      b < 1)
    b = 1;
  return b;
}

template <int CMAX, int W>
void launch_one(const BatchPass &bp, int sm_count, cudaStream_t s) {
  const size_t sm = smem_bytes<CMAX, W>(bp.blob_words);
  const int per = blocks_per_sm<CMAX, W>(sm);
  const uint64_t want = (bp.nblocks - bp.block_begin + W - 1) / W;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)per * sm_count));
  batch_kernel<CMAX, W><<<grid, W * 32, sm, s>>>(bp);
}

#include "batch4.cuh"
#include "batch_few.cuh"
#include "sparse_d2h.cuh"

template <int CMAX, int GV, int W>
size_t smem_bytes4(uint32_t blob_words) {
  return ((blob_words + 3) & ~3u) * 4 + (size_t)V4Shape<GV, W>::kStage * 4 + (size_t)kV4PosBytes<CMAX, GV, W>;
}

// Shared memory of a variant-4 pass: `groups` slot groups over up to `cmax`
// columns, blob of `blob_words` words, CTAs of `warps` warps.
size_t pass_smem4(size_t blob_words, int cmax, int groups, int warps) {
  const uint32_t w = (uint32_t)std::min<size_t>(blob_words, 1u << 30);
  if (warps == 8) {
    if (cmax <= 4)
      return groups == 4 ? smem_bytes4<4, 4, 8>(w) : groups == 8 ? smem_bytes4<4, 8, 8>(w) : smem_bytes4<4, 16, 8>(w);
    return groups == 4 ? smem_bytes4<8, 4, 8>(w) : groups == 8 ? smem_bytes4<8, 8, 8>(w) : smem_bytes4<8, 16, 8>(w);
  }
  if (cmax <= 4)
    return groups == 4 ? smem_bytes4<4, 4, 16>(w) : groups == 8 ? smem_bytes4<4, 8, 16>(w) : smem_bytes4<4, 16, 16>(w);
  return groups == 4 ? smem_bytes4<8, 4, 16>(w) : groups == 8 ? smem_bytes4<8, 8, 16>(w) : smem_bytes4<8, 16, 16>(w);
}

template <int CMAX, int GV, int W, bool PRE>
void launch_one4(const BatchPass &bp, int sm_count, cudaStream_t s) {
  static std::atomic<uint64_t> raised{0};
  raise_smem_limit(batch4_kernel<CMAX, GV, W, PRE>, raised, 227 * 1024);
  const size_t sm = smem_bytes4<CMAX, GV, W>(bp.blob_words);
  if (sm > 227 * 1024) throw Error(RTS_ERR_ARG, "batch pass exceeds shared memory");
  int per = 1;  // CTAs per SM: one, or two 8-warp CTAs when the shared memory holds both
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch4_kernel<CMAX, GV, W, PRE>, W * 32, sm) !=
          cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 1;
  }
  const uint64_t want = bp.nblocks - bp.block_begin;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count * per));
  batch4_kernel<CMAX, GV, W, PRE><<<grid, W * 32, sm, s>>>(bp);
}

template <int CMAX, int W>
void launch_shape4(const BatchPass &bp, int groups, int sm_count, cudaStream_t s) {
  if (groups == 16) launch_one4<CMAX, 16, W, false>(bp, sm_count, s);
  else if (groups == 8) launch_one4<CMAX, 8, W, false>(bp, sm_count, s);
  else launch_one4<CMAX, 4, W, false>(bp, sm_count, s);
}

// A pass fed by shared positions (256 or 512 slots, four columns or fewer).
void launch_pre4(const BatchPass &bp, int groups, int warps, int sm_count, cudaStream_t s) {
  if (warps == 8) {
    if (groups == 16) launch_one4<4, 16, 8, true>(bp, sm_count, s);
    else if (groups == 8) launch_one4<4, 8, 8, true>(bp, sm_count, s);
    else launch_one4<4, 4, 8, true>(bp, sm_count, s);
  } else {
    if (groups == 16) launch_one4<4, 16, 16, true>(bp, sm_count, s);
    else if (groups == 8) launch_one4<4, 8, 16, true>(bp, sm_count, s);
    else launch_one4<4, 4, 16, true>(bp, sm_count, s);
  }
}

// Rows per block of a variant-4 pass shape.
uint64_t rows_per_block4(int groups, int warps) {
  const int tiles_per_warp = 32 / groups;
  return (uint64_t)warps * tiles_per_warp * 32;
}

}  // namespace

// ---- host planning -----------------------------------------------------------

NormQuery normalize(const rts_term *terms, int n, int index, int ncols_table) {
  NormQuery q;
  q.index = index;
  SmallVec<int, 16> cols;
  SmallVec<uint32_t, 16> lo, hi;
  for (int i = 0; i < n; i++) {
    const rts_term &t = terms[i];
    if (t.column < 0 || t.column >= ncols_table) throw Error(RTS_ERR_ARG, "term column out of range");
    if (t.lo > t.hi) q.empty = true;
    const int *it = std::find(cols.begin(), cols.end(), (int)t.column);
    if (it == cols.end()) {
      cols.push_back(t.column);
      lo.push_back(t.lo);
      hi.push_back(t.hi);
    } else {
      const size_t k = it - cols.begin();
      lo[k] = std::max(lo[k], t.lo);
      hi[k] = std::min(hi[k], t.hi);
      if (lo[k] > hi[k]) q.empty = true;
    }
  }
  for (size_t k = 0; k < cols.size(); k++) {
    if (lo[k] == 0 && hi[k] == 0xFFFFFFFFu) continue;
    q.cols.push_back(cols[k]);
    q.lo.push_back(lo[k]);
    q.hi.push_back(hi[k]);
  }
  return q;
}

namespace {

// Distinct nonzero boundary values of one pass column: open addressing for
// membership, insertion order kept in `vals` (sorted when the pass closes).
// Boundaries are never 0 (a lower bound of 0 and an upper bound of 2^32 - 1
// constrain nothing), so 0 marks an empty cell.
struct BoundSet {
  std::vector<uint32_t> cell = std::vector<uint32_t>(64, 0u);
  std::vector<uint32_t> vals;
  uint32_t home(uint32_t v) const { return (v * 0x9E3779B1u) >> 7 & (uint32_t)(cell.size() - 1); }
  bool has(uint32_t v) const {
    for (uint32_t i = home(v);; i = (i + 1) & (uint32_t)(cell.size() - 1)) {
      if (cell[i] == v) return true;
      if (cell[i] == 0) return false;
    }
  }
  void add(uint32_t v) {
    if (has(v)) return;
    if (2 * (vals.size() + 1) > cell.size()) {
      cell.assign(cell.size() * 2, 0u);
      for (uint32_t x : vals) put(x);
    }
    put(v);
    vals.push_back(v);
  }
  size_t size() const { return vals.size(); }

 private:
  void put(uint32_t v) {
    uint32_t i = home(v);
    while (cell[i] != 0) i = (i + 1) & (uint32_t)(cell.size() - 1);
    cell[i] = v;
  }
};

struct PassPlan {
  std::vector<int> qs;              // normalized queries (indices into the list)
  std::vector<int> cols;            // table columns, in order
  std::vector<BoundSet> bounds;     // per table column
};

// Shared-memory bytes of a pass's tables, boundaries and bucket index for
// the given boundary counts (bucket index at most 4097 uint16 per column).
size_t column_bytes(size_t m, int G) {
  size_t nb = 1;
  while (nb < 4 * m && nb < 4096) nb <<= 1;
  return (m + 1) * (size_t)G * 4 + m * 4 + (nb + 2) * 2 + 8;
}

// Add query q to the pass if its tables still fit the budget (G words of
// 32 query bits per table row).
bool try_add(PassPlan &pp, const NormQuery &q, int qi, size_t budget, int max_per_pass, int G) {
  if ((int)pp.qs.size() >= std::min(max_per_pass, 32 * G)) return false;
  size_t total = 0;
  int new_cols = 0;
  size_t grow[kMaxCols] = {0};
  for (size_t k = 0; k < q.cols.size(); k++) {
    auto it = std::find(pp.cols.begin(), pp.cols.end(), q.cols[k]);
    size_t add = 0;
    if (it == pp.cols.end()) {
      new_cols++;
      add = (q.lo[k] > 0) + (q.hi[k] < 0xFFFFFFFFu);
      total += column_bytes(add, G);
    } else {
      const auto &S = pp.bounds[it - pp.cols.begin()];
      if (q.lo[k] > 0 && !S.has(q.lo[k])) grow[it - pp.cols.begin()]++;
      if (q.hi[k] < 0xFFFFFFFFu && !S.has(q.hi[k] + 1)) grow[it - pp.cols.begin()]++;
    }
  }
  if ((int)pp.cols.size() + new_cols > kMaxCols) return false;
  for (size_t c = 0; c < pp.cols.size(); c++) total += column_bytes(pp.bounds[c].size() + grow[c], G);
  if (total > budget && !pp.qs.empty()) return false;
  for (size_t k = 0; k < q.cols.size(); k++) {
    auto it = std::find(pp.cols.begin(), pp.cols.end(), q.cols[k]);
    size_t ci;
    if (it == pp.cols.end()) {
      pp.cols.push_back(q.cols[k]);
      pp.bounds.emplace_back();
      ci = pp.cols.size() - 1;
    } else {
      ci = it - pp.cols.begin();
    }
    if (q.lo[k] > 0) pp.bounds[ci].add(q.lo[k]);
    if (q.hi[k] < 0xFFFFFFFFu) pp.bounds[ci].add(q.hi[k] + 1);
  }
  pp.qs.push_back(qi);
  return true;
}

}  // namespace

// Device and pinned host buffers for batch plans, two of each so that the
// plan of the next batch can be built and uploaded while the previous batch
// still runs.
struct BatchScratch {
  struct Slot {
    void *dev = nullptr;
    size_t dev_cap = 0;
    uint32_t *host = nullptr;
    size_t host_cap = 0;
    cudaEvent_t done = nullptr;
  } slot[2];
  int next = 0;
  // shared positions of the context's batch calls: one buffer, and the
  // event after the last launch that reads it (a call on another stream
  // waits for it on the device)
  void *pre = nullptr;
  size_t pre_cap = 0;
  cudaEvent_t pre_done = nullptr;
  ~BatchScratch() {
    if (pre_done) cudaEventSynchronize(pre_done);
    if (pre) cudaFree(pre);
    if (pre_done) cudaEventDestroy(pre_done);
    for (auto &s : slot) {
      if (s.done) cudaEventSynchronize(s.done);
      if (s.dev) cudaFree(s.dev);
      if (s.host) cudaFreeHost(s.host);
      if (s.done) cudaEventDestroy(s.done);
    }
  }
};

void destroy_batch(BatchScratch *b) { delete b; }

// A planned batch: the mask-table passes of the queries that run in the
// kernel, built on the host once per query set.
struct BatchPlan {
  struct Pass {
    BatchPass bp;
    size_t off;  // word offset of the pass in `blob`
    int cmax;
    int variant;  // kernel the pass was planned for (3: 256-slot warps, 4: CTA-wide blocks)
    int warps;    // variant 4: warps per CTA the pass was planned for (8 or 16)
    int groups;   // 32-slot groups of the pass (table words per position)
    bool few;     // at most kFewMaxQueries queries: tested term by term (batch_few_kernel), no tables
    FewPass fp;
    int pre_slot = -1;  // shared positions: this pass's slot in the scratch, or -1 (it searches)
  };
  std::vector<Pass> passes;
  std::vector<uint32_t> blob;
  // shared positions of the passes with a pre_slot (npass 0: none)
  PreParams pre;
  size_t pre_off = 0;  // word offset of the union boundaries, buckets and maps in `blob`
  // batch_plan_drop: per query index, where its slot is (built at the first
  // drop): the blob word of a table-pass slot, or -(1 + pass) for a
  // term-by-term pass, or INT64_MIN when the plan does not hold it
  std::vector<int64_t> where;
};

// Answer the queries that do not run in the batch kernel (empty, no
// constrained column, more than eight constrained columns) over the whole
// table; returns the kernels launched.
int launch_outside(rts_ctx *ctx, const std::vector<NormQuery> &norm, const std::vector<int> &which,
                   const int32_t *out_index, uint32_t *out, uint64_t stride_words, unsigned long long *counts,
                   cudaStream_t s) {
  const uint64_t n = ctx->nrows;
  int launches = 0;
  for (int qi : which) {
    const NormQuery &q = norm[qi];
    const uint64_t o = out_index ? (uint64_t)out_index[qi] : (uint64_t)qi;
    uint32_t *bm = out + o * stride_words;
    if (q.empty || q.cols.empty()) {
      launch_fill_range(bm, n, !q.empty, counts + o, ctx->sm_count, s);
      launches += 1;
      continue;
    }
    ScanParams sp;
    memset(&sp, 0, sizeof sp);
    for (size_t first = 0; first < q.cols.size(); first += kFusedMaxTerms) {
      size_t cnt = std::min<size_t>(kFusedMaxTerms, q.cols.size() - first);
      bool vec = true;
      for (size_t i = 0; i < cnt; i++) {
        sp.t[i] = {ctx->cols[q.cols[first + i]], q.lo[first + i], q.hi[first + i] - q.lo[first + i]};
        vec = vec && (((uintptr_t)sp.t[i].col & 15) == 0);
      }
      sp.nterms = (int)cnt;
      sp.and_into = first > 0;
      sp.out = bm;
      sp.count = first + cnt == q.cols.size() ? counts + o : nullptr;
      sp.nrows = n;
      sp.full_tiles = n / kTileRows;
      if (first == 0) RTS_CUDA(cudaMemsetAsync(counts + o, 0, 8, s));
      launch_scan_fused(sp, vec, ctx->sm_count, s);
      launches++;
    }
  }
  return launches;
}

// Bucket index of a pass column's sorted boundaries B (B[0] = bmin, values
// up to bmin + span - 1): entry k is the first boundary in bucket k, so a
// value in bucket k only needs a search among B[bk[k] .. bk[k+1]).  Both the
// linear mapping (shift) and the log-linear one (bucket_of, mantissa bits
// *lgm) are built with at most nb_target buckets, and the one with the
// smaller mean search depth over the boundary intervals is kept (queries
// place their bounds at value quantiles, so each interval stands for about
// the same share of rows).  *lgm = 0 selects the linear mapping.
std::vector<uint16_t> bucket_index(const std::vector<uint32_t> &B, uint64_t span, uint32_t nb_target,
                                   uint32_t *shift_out, uint32_t *lgm_out) {
  const uint32_t m = (uint32_t)B.size(), bmin = B.front();
  // Search depth of the boundaries (all but the last) under a bucket map:
  // the sorted boundaries fall into non-decreasing buckets, so each run of
  // equal buckets is one bucket's boundaries (no index is built).
  auto depth = [&](auto &&bucket) {
    double d = 0;
    for (uint32_t lo = 0; lo < m;) {
      const uint32_t k = bucket(B[lo] - bmin);
      uint32_t hi = lo + 1;
      while (hi < m && bucket(B[hi] - bmin) == k) hi++;
      uint32_t it = 0;
      for (uint32_t n = hi - lo; n; n >>= 1) it++;
      d += (double)it * (hi - lo - (hi == m ? 1 : 0));
      lo = hi;
    }
    return d;
  };
  // the index of a bucket map over nb buckets: first boundary whose bucket is >= k
  auto index = [&](uint32_t nb, auto &&bucket) {
    std::vector<uint16_t> bk(nb + 1);
    uint32_t i = 0;
    for (uint32_t k = 0; k <= nb; k++) {
      while (i < m && bucket(B[i] - bmin) < k) i++;
      bk[k] = (uint16_t)i;
    }
    return bk;
  };
  uint32_t shift = 0;
  while ((span >> shift) > nb_target) shift++;
  const uint32_t nb = (uint32_t)(((span - 1) >> shift) + 1);  // buckets covering [bmin, bmax]
  auto lin = [&](uint32_t v) { return v >> shift; };
  *shift_out = shift;
  *lgm_out = 0;
  uint32_t M = 12;
  while (M > 0 && bucket_of((uint32_t)(span - 1), M) + 1 > nb_target) M--;
  if (M > 0) {
    auto lg = [&](uint32_t v) { return bucket_of(v, M); };
    if (depth(lg) < depth(lin)) {
      *lgm_out = M;
      return index(bucket_of((uint32_t)(span - 1), M) + 1, lg);
    }
  }
  return index(nb, lin);
}

bool runs_in_kernel(const NormQuery &q) { return !q.empty && !q.cols.empty() && (int)q.cols.size() <= kMaxCols; }

// Slot groups of a variant-4 pass of nq queries.
int pass_groups(int nq) { return nq <= 128 ? 4 : nq <= 256 ? 8 : 16; }

// Start of bucket k of a union column, relative to its origin (inverse of
// pre_bucket below the clamp).
uint64_t pre_bucket_start(uint32_t M, uint32_t L, uint32_t k) {
  if ((k >> M) <= 1) return (uint64_t)k << L;  // linear part
  const uint32_t t = (k >> M) - 1;
  const uint64_t w = (k & ((1u << M) - 1)) | (1u << M);
  return w << (t + L);
}

// Bucket index of a union column (PreCol) with at most kPreMaxBuckets
// buckets.  Candidates: linear buckets, and for M = 1..12 the log-linear
// ones with the smallest L that fits; the one whose boundaries need the
// fewest search steps in all wins (the query bounds sit where the rows
// are dense), fewer buckets on a tie.
std::vector<uint32_t> pre_buckets(const std::vector<uint32_t> &B, PreCol &pc) {
  const uint32_t m = (uint32_t)B.size();
  pc.m = m;
  pc.origin = m && B[0] > 0 ? B[0] - 1 : 0;
  if (m == 0) {
    pc.M = 31;
    pc.L = 0;
    pc.nbk = 1;
    return {0u};
  }
  // Search steps of every boundary under bucket shape (M, L): the sorted
  // boundaries fall into non-decreasing buckets, so each run of equal
  // buckets is one bucket's boundaries (no index is built).
  auto cost_of = [&](uint32_t M, uint32_t L, uint32_t nbk) {
    PreCol t = pc;
    t.M = M;
    t.L = L;
    t.nbk = nbk;
    double cost = 0;
    auto close = [&](uint32_t k, uint32_t lo, uint32_t hi) {  // boundaries [lo, hi) in bucket k
      const uint64_t start = (uint64_t)pc.origin + pre_bucket_start(M, L, k);
      const uint32_t n = hi - lo - (B[lo] == start ? 1u : 0u);
      uint32_t steps = 0;
      for (uint32_t r = n; r; r >>= 1) steps++;
      cost += (double)steps * (hi - lo);
    };
    uint32_t lo = 0, k = pre_bucket(t, B[0]);
    for (uint32_t i = 1; i < m; i++) {
      const uint32_t ki = pre_bucket(t, B[i]);
      if (ki != k) {
        close(k, lo, i);
        lo = i;
        k = ki;
      }
    }
    close(k, lo, m);
    return cost;
  };
  const uint32_t vmax = B.back() - pc.origin;
  uint32_t bestM, bestL, bestN;
  {
    uint32_t L = 0;
    while ((vmax >> L) >= kPreMaxBuckets) L++;
    bestM = 31;
    bestL = L;
    bestN = (vmax >> L) + 1;
  }
  double best_cost = cost_of(bestM, bestL, bestN);
  for (uint32_t M = 1; M <= 12; M++)
    for (uint32_t L = 0; L < 32; L++) {
      PreCol t = pc;
      t.M = M;
      t.L = L;
      t.nbk = 0xFFFFFFFFu;
      const uint32_t nbk = pre_bucket(t, B.back()) + 1;
      if (nbk > kPreMaxBuckets) continue;
      const double cost = cost_of(M, L, nbk);
      if (cost < best_cost || (cost == best_cost && nbk < bestN)) {
        best_cost = cost;
        bestM = M;
        bestL = L;
        bestN = nbk;
      }
      break;
    }
  pc.M = bestM;
  pc.L = bestL;
  pc.nbk = bestN;
  // the index: entry k = base | n << 16 (see PreCol)
  std::vector<uint32_t> ent(bestN);
  uint32_t lo = 0;
  for (uint32_t k = 0; k < bestN; k++) {
    uint32_t hi = lo;
    while (hi < m && (k + 1 == bestN || pre_bucket(pc, B[hi]) == k)) hi++;
    const uint64_t start = (uint64_t)pc.origin + pre_bucket_start(bestM, bestL, k);
    const uint32_t base = lo + (lo < hi && B[lo] == start ? 1u : 0u);
    ent[k] = base | (hi - base) << 16;
    lo = hi;
  }
  return ent;
}

// Move column s of `src` to column c of `dst` (a pass's per-column fields).
void move_column(BatchPass &dst, int c, const BatchPass &src, int s) {
  dst.col[c] = src.col[s];
  dst.m[c] = src.m[s];
  dst.bmin[c] = src.bmin[s];
  dst.bmax[c] = src.bmax[s];
  dst.shift[c] = src.shift[s];
  dst.lgm[c] = src.lgm[s];
  dst.tab_off[c] = src.tab_off[s];
  dst.bnd_off[c] = src.bnd_off[s];
  dst.bkt_off[c] = src.bkt_off[s];
  dst.nbk[c] = src.nbk[s];
}

// Shared positions for a plan with one or more table passes of the
// look-ahead shapes (256 or 512 slots, at most four columns) over the same
// columns (one pass too: on 1e8 rows x 4 columns the pre-pass and a pass
// reading positions took 2.08 ms for 256 queries and 3.44 ms for 512,
// against 2.67 and 3.98 ms for the pass that searches): the later passes' columns are put in the first one's order; per
// column the union of the passes' boundaries with its bucket index, and
// the map from a union position to every pass's table word offset (a
// pass's boundaries are a subset of the union, so the pass position of
// union position k is the number of its boundaries <= B_u[k-1]).  Appended
// to the plan blob; other plans are left as they are.
void plan_shared_positions(BatchPlan &plan) {
  plan.pre.npass = 0;
  std::vector<int> which;
  for (size_t i = 0; i < plan.passes.size() && (int)which.size() < kMaxPrePasses; i++) {
    const BatchPlan::Pass &b = plan.passes[i];
    if (b.few || b.variant != 4 || b.cmax != 4) continue;
    if (!which.empty()) {
      const BatchPass &f = plan.passes[which[0]].bp;
      if (b.bp.ncols != f.ncols) continue;
      bool same = true;
      for (int c = 0; c < f.ncols; c++) same = same && std::find(b.bp.col, b.bp.col + b.bp.ncols, f.col[c]) != b.bp.col + b.bp.ncols;
      if (!same) continue;
    }
    which.push_back((int)i);
  }
  if (which.empty()) return;
  const int U = plan.passes[which[0]].bp.ncols;
  const int npass = (int)which.size(), NW = (npass + 1) / 2;
  std::vector<std::vector<uint32_t>> Bu(U);
  std::vector<BatchPass> ordered(npass);
  for (int q = 0; q < npass; q++) {
    const BatchPass &src = plan.passes[which[q]].bp;
    ordered[q] = src;
    for (int c = 0; c < U; c++) {
      const int s = (int)(std::find(src.col, src.col + U, plan.passes[which[0]].bp.col[c]) - src.col);
      move_column(ordered[q], c, src, s);
    }
    // each pass's boundaries are sorted: merge them into the union
    const uint32_t *blob = plan.blob.data() + plan.passes[which[q]].off;
    for (int c = 0; c < U; c++) {
      const uint32_t *Bp = blob + ordered[q].bnd_off[c];
      std::vector<uint32_t> merged(Bu[c].size() + ordered[q].m[c]);
      merged.resize(std::set_union(Bu[c].begin(), Bu[c].end(), Bp, Bp + ordered[q].m[c], merged.begin()) -
                    merged.begin());
      Bu[c].swap(merged);
    }
  }
  PreParams P;
  memset(&P, 0, sizeof P);
  P.ncols = U;
  P.npass = npass;
  std::vector<uint32_t> ub;  // offsets relative to its own start
  for (int c = 0; c < U; c++) {
    const std::vector<uint32_t> &B = Bu[c];  // sorted and distinct
    if (B.size() > 0xFFFFu) return;  // bucket entries hold 16-bit positions
    PreCol &pc = P.c[c];
    pc.col = ordered[0].col[c];
    const std::vector<uint32_t> ent = pre_buckets(B, pc);
    pc.bkt_off = (uint32_t)ub.size();
    ub.insert(ub.end(), ent.begin(), ent.end());
    pc.bnd_off = (uint32_t)ub.size();
    ub.insert(ub.end(), B.begin(), B.end());
    if (NW == 2 && ub.size() % 2) ub.push_back(0);  // 8-byte map entries
    pc.map_off = (uint32_t)ub.size();
    ub.resize(ub.size() + (B.size() + 1) * NW, 0u);
    for (int q = 0; q < npass; q++) {
      const BatchPlan::Pass &b = plan.passes[which[q]];
      const uint32_t *Bp = plan.blob.data() + b.off + ordered[q].bnd_off[c];
      const uint32_t mp = ordered[q].m[c];
      uint32_t j = 0;
      for (size_t k = 0; k <= B.size(); k++) {
        if (k > 0)
          while (j < mp && Bp[j] <= B[k - 1]) j++;
        const uint64_t off = (uint64_t)ordered[q].tab_off[c] + (uint64_t)j * b.groups;
        if (off > 0xFFFFu) return;  // table offsets are 16-bit in the map
        ub[pc.map_off + k * NW + q / 2] |= (uint32_t)off << (16 * (q & 1));
      }
    }
  }
  if (ub.size() * 4 > 200 * 1024) return;  // the pre kernel's shared memory
  P.blob_words = (uint32_t)ub.size();
  plan.pre = P;
  for (int q = 0; q < npass; q++) {
    plan.passes[which[q]].bp = ordered[q];
    plan.passes[which[q]].pre_slot = q;
  }
  while (plan.blob.size() % 4) plan.blob.push_back(0);
  plan.pre_off = plan.blob.size();
  plan.blob.insert(plan.blob.end(), ub.begin(), ub.end());
}

// Passes for the kernel queries `which` (indices into norm); query qi writes
// bitmap out_index[qi] (qi when null).
BatchPlan build_plan(rts_ctx *ctx, const std::vector<NormQuery> &norm, const std::vector<int> &which,
                     const int32_t *out_index, size_t table_budget, bool share_positions) {
  const int variant = ctx->batch_cfg.variant == 4 ? 4 : 3;
  const int warps4 = ctx->batch_cfg.warps_per_cta == 8 ? 8 : 16;
  const int G = variant == 4 ? 16 : kGroups;  // pass capacity in groups (budgeted at this table width)
  std::vector<PassPlan> passes;
  for (int qi : which) {
    const int per = ctx->batch_cfg.max_queries_per_pass;
    if (passes.empty() || !try_add(passes.back(), norm[qi], qi, table_budget, per, G)) {
      passes.emplace_back();
      if (!try_add(passes.back(), norm[qi], qi, table_budget, per, G))
        throw Error(RTS_ERR_ARG, "query does not fit one batch pass");
    }
  }
  BatchPlan plan;
  for (auto &pp : passes) {
    BatchPlan::Pass b;
    memset(&b.bp, 0, sizeof b.bp);
    memset(&b.fp, 0, sizeof b.fp);
    b.few = false;
    const int C = (int)pp.cols.size();
    if (variant == 4 && (int)pp.qs.size() <= kFewMaxQueries) {
      FewPass &fp = b.fp;
      b.few = true;
      b.variant = variant;
      b.warps = warps4;
      b.groups = 1;
      b.cmax = C <= 4 ? 4 : 8;
      fp.nq = (int)pp.qs.size();
      fp.ncols = C;
      for (int c = 0; c < C; c++) fp.col[c] = ctx->cols[pp.cols[c]];
      for (int j = 0; j < kFewSlots; j++) {
        fp.slot_query[j] = -1;
        for (int c = 0; c < kMaxCols; c++) fp.term[j][c] = make_uint2(0u, 0xFFFFFFFFu);  // always true
      }
      for (int j = 0; j < fp.nq; j++) {
        const NormQuery &q = norm[pp.qs[j]];
        fp.slot_query[j] = out_index ? out_index[pp.qs[j]] : pp.qs[j];
        for (size_t k = 0; k < q.cols.size(); k++) {
          const int c = (int)(std::find(pp.cols.begin(), pp.cols.end(), q.cols[k]) - pp.cols.begin());
          fp.term[j][c] = make_uint2(q.lo[k], q.hi[k] - q.lo[k]);
        }
      }
      b.off = plan.blob.size();
      plan.passes.push_back(b);
      continue;
    }
    BatchPass &bp = b.bp;
    // 4: the smallest of the 128-, 256- and 512-slot shapes that holds the pass
    const int Gp = variant == 4 ? pass_groups((int)pp.qs.size()) : kGroups;
    b.groups = Gp;
    bp.ncols = C;
    std::vector<uint32_t> blob;
    std::vector<std::vector<uint32_t>> B(C);
    for (int c = 0; c < C; c++) {
      B[c] = std::move(pp.bounds[c].vals);
      std::sort(B[c].begin(), B[c].end());
      bp.m[c] = (uint32_t)B[c].size();
    }
    // tables: row pos holds, per slot, whether the values of interval pos
    // ([B[pos-1], B[pos]) with B[-1] = 0, B[m] = 2^32) pass the slot's term
    // on this column (always, when the slot does not constrain it).  Built
    // in place as XOR deltas at the interval ends and a prefix XOR over
    // positions; a term [lo, hi] covers positions pos(lo) .. pos(hi) with
    // pos(x) = #{B <= x}, where lo and hi + 1 are themselves boundaries.
    for (int c = 0; c < C; c++) {
      bp.tab_off[c] = (uint32_t)blob.size();
      blob.resize(blob.size() + (size_t)(bp.m[c] + 1) * Gp, 0u);
    }
    std::vector<uint32_t> free_mask((size_t)C * Gp, 0u);  // slots leaving column c unconstrained
    for (int slot = 0; slot < (int)pp.qs.size(); slot++) {
      const uint32_t bit = 1u << (slot & 31);
      const int grp = slot >> 5;
      for (int c = 0; c < C; c++) free_mask[(size_t)c * Gp + grp] |= bit;
      const NormQuery &q = norm[pp.qs[slot]];
      for (size_t k = 0; k < q.cols.size(); k++) {
        const int c = (int)(std::find(pp.cols.begin(), pp.cols.end(), q.cols[k]) - pp.cols.begin());
        const std::vector<uint32_t> &Bc = B[c];
        const uint32_t m = bp.m[c];
        const uint32_t p0 =
            q.lo[k] > 0 ? (uint32_t)(std::lower_bound(Bc.begin(), Bc.end(), q.lo[k]) - Bc.begin()) + 1 : 0u;
        const uint32_t p1 = q.hi[k] < 0xFFFFFFFFu
                                ? (uint32_t)(std::lower_bound(Bc.begin(), Bc.end(), q.hi[k] + 1) - Bc.begin())
                                : m;
        uint32_t *tab = blob.data() + bp.tab_off[c];
        tab[(size_t)p0 * Gp + grp] ^= bit;
        if (p1 + 1 <= m) tab[(size_t)(p1 + 1) * Gp + grp] ^= bit;
        free_mask[(size_t)c * Gp + grp] &= ~bit;
      }
    }
    for (int c = 0; c < C; c++) {
      uint32_t *tab = blob.data() + bp.tab_off[c];
      for (int grp = 0; grp < Gp; grp++) tab[grp] ^= free_mask[(size_t)c * Gp + grp];  // pass every position
      for (size_t i = Gp; i < (size_t)(bp.m[c] + 1) * Gp; i++) tab[i] ^= tab[i - Gp];
    }
    // boundaries and bucket index.  The table budget counts 4 buckets per
    // boundary; a pass takes 16 where its shared memory still holds them:
    // fewer boundaries per bucket make more loop-free lookups exact and the
    // searches shorter.
    auto buckets_for = [](uint32_t m, uint32_t per) {
      uint32_t nb = 1;
      while (nb < per * m && nb < 4096) nb <<= 1;
      return nb;
    };
    uint32_t per = 4;
    if (variant == 4) {
      size_t w = blob.size() + 32 * (size_t)Gp;  // tables so far, slot map
      for (int c = 0; c < C; c++) w += bp.m[c] + (bp.m[c] ? (buckets_for(bp.m[c], 16) + 3) / 2 : 1);
      if (pass_smem4(w, C <= 4 ? 4 : 8, Gp, warps4) <= 227 * 1024) per = 16;
    }
    for (int c = 0; c < C; c++) {
      const uint32_t m = bp.m[c];
      bp.bnd_off[c] = (uint32_t)blob.size();
      blob.insert(blob.end(), B[c].begin(), B[c].end());
      if (m == 0) {
        bp.bkt_off[c] = (uint32_t)blob.size();
        bp.nbk[c] = 1;
        blob.push_back(0);
        continue;
      }
      bp.bmin[c] = B[c].front();
      bp.bmax[c] = B[c].back();
      const uint64_t span = (uint64_t)bp.bmax[c] - bp.bmin[c] + 1;
      const std::vector<uint16_t> bk = bucket_index(B[c], span, buckets_for(m, per), &bp.shift[c], &bp.lgm[c]);
      bp.nbk[c] = (uint32_t)bk.size() - 1;
      bp.bkt_off[c] = (uint32_t)blob.size();
      const size_t wsz = (bk.size() + 1) / 2;
      blob.resize(blob.size() + wsz, 0u);
      memcpy(blob.data() + bp.bkt_off[c], bk.data(), bk.size() * 2);
    }
    bp.slot_off = (uint32_t)blob.size();
    for (int slot = 0; slot < 32 * Gp; slot++) {
      uint32_t o = 0xFFFFFFFFu;
      if (slot < (int)pp.qs.size()) o = out_index ? (uint32_t)out_index[pp.qs[slot]] : (uint32_t)pp.qs[slot];
      blob.push_back(o);
    }
    bp.blob_words = (uint32_t)blob.size();
    for (int c = 0; c < C; c++) bp.col[c] = ctx->cols[pp.cols[c]];
    b.cmax = C <= 4 ? 4 : 8;
    b.variant = variant;
    b.warps = warps4;
    while (plan.blob.size() % 4) plan.blob.push_back(0);  // 16-byte aligned pass start
    b.off = plan.blob.size();
    plan.blob.insert(plan.blob.end(), blob.begin(), blob.end());
    plan.passes.push_back(b);
  }
  if (share_positions) plan_shared_positions(plan);
  return plan;
}

// A term-by-term pass slot's term on a column it does not constrain.
bool always_true(uint2 term) { return term.x == 0 && term.y == 0xFFFFFFFFu; }

// Whether a term-by-term pass runs as one fused scan per query instead: one
// query always; two or three when they have at most six terms between them.
// On a 2^23-row segment of 4 columns a fused scan takes about 5.6 us plus
// 5.9 us per term; two queries of 1, 2 and 3 columns each took 17, 28 and
// 41 us as fused scans against 27, 50 and 54 us term by term (4 columns
// each: 55 us either way).
bool fused_each(const FewPass &f) {
  if (f.nq > 3) return false;
  int terms = 0;
  for (int j = 0; j < f.nq; j++) {
    int k = 0;
    for (int c = 0; c < f.ncols; c++) k += !always_true(f.term[j][c]);
    if (k == 0) return false;  // (no such slot reaches a pass; the kernel would answer it)
    terms += k;
  }
  return f.nq == 1 || terms <= 6;
}

// The pre kernel over P's rows, one block per SM and resident slot.
template <int U, int NW>
void launch_pre_shape(rts_ctx *ctx, const PreParams &P, cudaStream_t s) {
  static std::atomic<uint64_t> raised{0};
  raise_smem_limit(pre_kernel<U, NW>, raised, 227 * 1024);
  const size_t sm = (size_t)P.blob_words * 4;
  int per = 1;  // resident blocks per SM with this blob
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pre_kernel<U, NW>, kPreThreads, sm) != cudaSuccess ||
      per < 1) {
    cudaGetLastError();
    per = 1;
  }
  const uint64_t blocks = (P.row_end - P.row_begin + kPreTile - 1) / kPreTile;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)ctx->sm_count * per));
  pre_kernel<U, NW><<<grid, kPreThreads, sm, s>>>(P);
}

template <int NW>
void launch_pre_nw(rts_ctx *ctx, const PreParams &P, cudaStream_t s) {
  switch (P.ncols) {
    case 1: launch_pre_shape<1, NW>(ctx, P, s); break;
    case 2: launch_pre_shape<2, NW>(ctx, P, s); break;
    case 3: launch_pre_shape<3, NW>(ctx, P, s); break;
    default: launch_pre_shape<4, NW>(ctx, P, s); break;
  }
}

void launch_pre(rts_ctx *ctx, PreParams P, cudaStream_t s) {
  P.stride = pre_stride(P.row_end - P.row_begin);
  P.vec = ((uintptr_t)P.out & 15) == 0;
  for (int c = 0; c < P.ncols; c++) P.vec = P.vec && ((uintptr_t)(P.c[c].col + P.row_begin) & 7) == 0;
  if (P.npass <= 2)
    launch_pre_nw<1>(ctx, P, s);
  else
    launch_pre_nw<2>(ctx, P, s);
}

// Launch every pass of `plan` (blob already on the device) over rows
// [row_begin, row_end); row_begin is a multiple of 4096 (the largest block
// of the pass shapes).  Returns launches.
int launch_plan(rts_ctx *ctx, BatchPlan &plan, const uint32_t *dev_blob, uint32_t *out, uint64_t stride_words,
                unsigned long long *counts, uint64_t row_begin, uint64_t row_end, void *scratch,
                size_t scratch_bytes, cudaStream_t s) {
  int launches = 0;
  // shared positions, when the caller's scratch holds them; else every pass
  // searches its own
  const uint64_t pre_rows = row_end > row_begin ? row_end - row_begin : 0;
  const bool pre = plan.pre.npass > 0 && pre_rows > 0 && scratch &&
                   (uint64_t)plan.pre.npass * pre_stride(pre_rows) * sizeof(uint2) <= scratch_bytes;
  if (pre) {
    PreParams P = plan.pre;
    P.blob = dev_blob + plan.pre_off;
    P.row_begin = row_begin;
    P.row_end = row_end;
    P.out = static_cast<uint2 *>(scratch);
    launch_pre(ctx, P, s);
    launches++;
  }
  for (auto &b : plan.passes) {
    if (b.few && fused_each(b.fp)) {
      // one query (or two over few columns): the single-query scan kernel
      // over the range per query, which runs at HBM speed (the term-by-term
      // kernel reaches about half of it here); the range starts at a
      // multiple of 4096 rows, so the column and bitmap offsets keep their
      // alignment, and the counts accumulate
      const FewPass &f = b.fp;
      for (int j = 0; j < f.nq; j++) {
        if (f.slot_query[j] < 0) continue;
        ScanParams sp;
        memset(&sp, 0, sizeof sp);
        bool vec = true;
        for (int c = 0; c < f.ncols; c++) {
          if (always_true(f.term[j][c])) continue;
          DevTerm &dt = sp.t[sp.nterms++];
          dt = {f.col[c] + row_begin, f.term[j][c].x, f.term[j][c].y};
          vec = vec && (((uintptr_t)dt.col & 15) == 0);
        }
        sp.out = out + (uint64_t)f.slot_query[j] * stride_words + row_begin / 32;
        sp.count = counts + f.slot_query[j];
        sp.nrows = row_end - row_begin;
        sp.full_tiles = sp.nrows / kTileRows;
        launch_scan_fused(sp, vec, ctx->sm_count, s);
        launches++;
      }
      continue;
    }
    if (b.few) {
      FewPass fp = b.fp;
      fp.out = out;
      fp.stride_words = stride_words;
      fp.counts = counts;
      fp.nrows = row_end;
      fp.words = words_for(ctx->nrows);
      fp.tile_begin = row_begin / 1024;
      fp.ntiles = (row_end + 1023) / 1024;
      const uint64_t ctas = (fp.ntiles - fp.tile_begin + kFewWarps - 1) / kFewWarps;
      const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(ctas, (uint64_t)ctx->sm_count * 8));
      switch (fp.ncols) {
        case 1: launch_few<1>(fp, grid, s); break;
        case 2: launch_few<2>(fp, grid, s); break;
        case 3: launch_few<3>(fp, grid, s); break;
        case 4: launch_few<4>(fp, grid, s); break;
        case 5: launch_few<5>(fp, grid, s); break;
        case 6: launch_few<6>(fp, grid, s); break;
        case 7: launch_few<7>(fp, grid, s); break;
        default: launch_few<8>(fp, grid, s); break;
      }
      launches++;
      continue;
    }
    const uint64_t rows_per_block =
        b.variant != 4 ? (uint64_t)(32 * kTilesPerBlock) : rows_per_block4(b.groups, b.warps);
    BatchPass bp = b.bp;
    bp.blob = dev_blob + b.off;
    bp.out = out;
    bp.stride_words = stride_words;
    bp.counts = counts;
    bp.nrows = row_end;
    bp.words = words_for(ctx->nrows);
    bp.block_begin = row_begin / rows_per_block;
    bp.nblocks = (row_end + rows_per_block - 1) / rows_per_block;
    bp.vec_store = (((uintptr_t)out & 15) == 0 && stride_words % 4 == 0) ? 1 : 0;
    bp.word_bytes = 4;
    const bool w8 = ctx->batch_cfg.warps_per_cta == 8;
    if (pre && b.pre_slot >= 0) {
      bp.pre = static_cast<const uint2 *>(scratch) + (uint64_t)b.pre_slot * pre_stride(pre_rows);
      bp.pre_row0 = row_begin;
      launch_pre4(bp, b.groups, b.warps, ctx->sm_count, s);
    } else if (b.variant == 4) {
      if (b.cmax == 4) {
        if (b.warps == 8) launch_shape4<4, 8>(bp, b.groups, ctx->sm_count, s);
        else launch_shape4<4, 16>(bp, b.groups, ctx->sm_count, s);
      } else {
        if (b.warps == 8) launch_shape4<8, 8>(bp, b.groups, ctx->sm_count, s);
        else launch_shape4<8, 16>(bp, b.groups, ctx->sm_count, s);
      }
    } else if (b.cmax == 4) {
      if (w8) launch_one<4, 8>(bp, ctx->sm_count, s);
      else launch_one<4, 16>(bp, ctx->sm_count, s);
    } else {
      if (w8) launch_one<8, 8>(bp, ctx->sm_count, s);
      else launch_one<8, 16>(bp, ctx->sm_count, s);
    }
    launches++;
  }
  return launches;
}

std::vector<NormQuery> normalize_all(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int nq) {
  std::vector<NormQuery> norm;
  norm.reserve(nq);
  for (int q = 0; q < nq; q++) {
    if (offsets[q + 1] < offsets[q] || offsets[q] < 0) throw Error(RTS_ERR_ARG, "offsets not ascending");
    norm.push_back(normalize(terms + offsets[q], offsets[q + 1] - offsets[q], q, (int)ctx->cols.size()));
  }
  return norm;
}

// Copy `plan` to one of the context's two plan buffers (pinned staging +
// device), waiting for the batch that used that buffer two calls ago.
const uint32_t *upload_plan(rts_ctx *ctx, const BatchPlan &plan, cudaStream_t s, cudaEvent_t *done) {
  if (!ctx->batch) ctx->batch = new BatchScratch();
  BatchScratch::Slot &S = ctx->batch->slot[ctx->batch->next];
  ctx->batch->next ^= 1;
  const size_t bytes = std::max<size_t>(plan.blob.size(), 4) * 4;
  if (S.done) RTS_CUDA(cudaEventSynchronize(S.done));
  else RTS_CUDA(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming));
  if (S.dev_cap < bytes) {
    if (S.dev) cudaFree(S.dev);
    S.dev = nullptr;
    S.dev_cap = 0;
    if (cudaMalloc(&S.dev, bytes) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "batch plan allocation failed");
    }
    S.dev_cap = bytes;
  }
  if (S.host_cap < bytes) {
    if (S.host) cudaFreeHost(S.host);
    S.host = nullptr;
    S.host_cap = 0;
    RTS_CUDA(cudaMallocHost(&S.host, bytes));
    S.host_cap = bytes;
  }
  memcpy(S.host, plan.blob.data(), plan.blob.size() * 4);
  RTS_CUDA(cudaMemcpyAsync(S.dev, S.host, plan.blob.size() * 4, cudaMemcpyHostToDevice, s));
  *done = S.done;
  return reinterpret_cast<const uint32_t *>(S.dev);
}

size_t plan_pre_bytes(const BatchPlan &plan, uint64_t rows) {
  return (size_t)plan.pre.npass * pre_stride(rows) * sizeof(uint2);
}

// The context's shared-position scratch for `bytes`, ordered after its last
// use on stream s; null (the passes then search) when the plan needs none or
// the device has no room (at most an eighth of it is used).
void *context_pre_scratch(rts_ctx *ctx, size_t bytes, cudaStream_t s) {
  if (!bytes) return nullptr;
  if (!ctx->batch) ctx->batch = new BatchScratch();
  BatchScratch &B = *ctx->batch;
  if (!B.pre_done) RTS_CUDA(cudaEventCreateWithFlags(&B.pre_done, cudaEventDisableTiming));
  if (B.pre_cap < bytes) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || bytes > total_b / 8) {
      cudaGetLastError();
      return nullptr;
    }
    RTS_CUDA(cudaEventSynchronize(B.pre_done));
    if (B.pre) cudaFree(B.pre);
    B.pre = nullptr;
    B.pre_cap = 0;
    if (cudaMalloc(&B.pre, bytes) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    B.pre_cap = bytes;
  }
  RTS_CUDA(cudaStreamWaitEvent(s, B.pre_done, 0));
  return B.pre;
}

void context_pre_done(rts_ctx *ctx, cudaStream_t s) {
  if (ctx->batch && ctx->batch->pre_done) RTS_CUDA(cudaEventRecord(ctx->batch->pre_done, s));
}

void batch_scan(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int nq, uint32_t *out,
                uint64_t stride_words, unsigned long long *counts, cudaStream_t s, size_t table_budget) {
  std::vector<NormQuery> norm = normalize_all(ctx, terms, offsets, nq);
  std::vector<int> inside, outside;
  for (int q = 0; q < nq; q++) (runs_in_kernel(norm[q]) ? inside : outside).push_back(q);
  // every count starts at zero; the kernel accumulates, fills overwrite
  RTS_CUDA(cudaMemsetAsync(counts, 0, (size_t)nq * 8, s));
  int launches = launch_outside(ctx, norm, outside, nullptr, out, stride_words, counts, s);
  if (!inside.empty()) {
    BatchPlan plan = build_plan(ctx, norm, inside, nullptr, table_budget, true);
    cudaEvent_t done = nullptr;
    const uint32_t *dev_blob = upload_plan(ctx, plan, s, &done);
    const size_t pre_bytes = plan_pre_bytes(plan, ctx->nrows);
    void *pre = context_pre_scratch(ctx, pre_bytes, s);
    launches += launch_plan(ctx, plan, dev_blob, out, stride_words, counts, 0, ctx->nrows, pre, pre_bytes, s);
    if (pre) context_pre_done(ctx, s);
    RTS_CUDA(cudaEventRecord(done, s));
  }
  RTS_CUDA(cudaGetLastError());
  ctx->launches += launches;
}

void BatchPlanDeleter::operator()(BatchPlan *p) const { delete p; }

BatchPlanPtr make_batch_plan(rts_ctx *ctx, const std::vector<NormQuery> &norm, const std::vector<int> &which,
                             const int32_t *out_index, size_t table_budget, bool share_positions) {
  return BatchPlanPtr(new BatchPlan(build_plan(ctx, norm, which, out_index, table_budget, share_positions)));
}

const std::vector<uint32_t> &batch_plan_blob(const BatchPlan &plan) { return plan.blob; }

void batch_plan_drop(BatchPlan &plan, int qi, std::vector<uint32_t> &blob_words) {
  if (plan.where.empty()) {
    int maxq = 0;
    for (const auto &b : plan.passes) {
      if (b.few) {
        for (int j = 0; j < b.fp.nq; j++) maxq = std::max(maxq, b.fp.slot_query[j]);
      } else {
        const int32_t *slot = reinterpret_cast<const int32_t *>(plan.blob.data() + b.off + b.bp.slot_off);
        for (int sl = 0; sl < 32 * b.groups; sl++) maxq = std::max(maxq, slot[sl]);
      }
    }
    plan.where.assign((size_t)maxq + 1, INT64_MIN);
    for (size_t i = 0; i < plan.passes.size(); i++) {
      const auto &b = plan.passes[i];
      if (b.few) {
        for (int j = 0; j < b.fp.nq; j++)
          if (b.fp.slot_query[j] >= 0) plan.where[b.fp.slot_query[j]] = -1 - (int64_t)i;
      } else {
        const size_t base = b.off + b.bp.slot_off;
        const int32_t *slot = reinterpret_cast<const int32_t *>(plan.blob.data() + base);
        for (int sl = 0; sl < 32 * b.groups; sl++)
          if (slot[sl] >= 0) plan.where[slot[sl]] = (int64_t)(base + sl);
      }
    }
  }
  if (qi < 0 || (size_t)qi >= plan.where.size() || plan.where[qi] == INT64_MIN) return;
  const int64_t w = plan.where[qi];
  plan.where[qi] = INT64_MIN;
  if (w >= 0) {
    plan.blob[w] = 0xFFFFFFFFu;
    blob_words.push_back((uint32_t)w);
    return;
  }
  FewPass &f = plan.passes[(size_t)(-1 - w)].fp;
  for (int j = 0; j < f.nq; j++)
    if (f.slot_query[j] == qi) f.slot_query[j] = -1;
}

int launch_batch_plan(rts_ctx *ctx, BatchPlan &plan, const uint32_t *dev_blob, uint32_t *out, uint64_t stride_words,
                      unsigned long long *counts, uint64_t row_begin, uint64_t row_end, void *scratch,
                      size_t scratch_bytes, cudaStream_t s) {
  return launch_plan(ctx, plan, dev_blob, out, stride_words, counts, row_begin, row_end, scratch, scratch_bytes, s);
}

size_t batch_plan_scratch_bytes(const BatchPlan &plan, uint64_t rows) { return plan_pre_bytes(plan, rows); }

}  // namespace rts

namespace rts {
// Device buffers of the host-buffer batch call, kept by the context.
struct HostBatchBuffers {
  uint32_t *cols = nullptr;
  size_t cols_cap = 0;
  uint32_t *bitmaps = nullptr;
  size_t bm_cap = 0;
  unsigned long long *counts = nullptr;
  size_t cnt_cap = 0;
  cudaStream_t up = nullptr, compute = nullptr, copy = nullptr;
  std::vector<cudaEvent_t> ev;
  // sparse transfer: per chunk the queries' nonzero-word counts (device,
  // pinned host), the packed queries and their pair offsets (pinned host,
  // device), and the packed chunks (two device slots, three pinned host slots)
  uint32_t *nnz = nullptr;
  size_t nnz_cap = 0;
  uint32_t *nnz_host = nullptr;
  size_t nnz_host_cap = 0;
  int32_t *ql = nullptr;
  size_t ql_cap = 0;
  uint64_t *qoff = nullptr;
  size_t qoff_cap = 0;
  int32_t *ql_host = nullptr;
  size_t ql_host_cap = 0;
  uint64_t *qoff_host = nullptr;
  size_t qoff_host_cap = 0;
  uint32_t *packed[2] = {nullptr, nullptr};
  size_t packed_cap[2] = {0, 0};
  uint32_t *packed_host[3] = {nullptr, nullptr, nullptr};
  size_t packed_host_cap[3] = {0, 0, 0};
  // bytes the last call moved each way
  uint64_t last_h2d = 0, last_d2h = 0;
  ~HostBatchBuffers() {
    if (up) cudaStreamSynchronize(up);
    if (compute) cudaStreamSynchronize(compute);
    if (copy) cudaStreamSynchronize(copy);
    if (cols) cudaFree(cols);
    if (bitmaps) cudaFree(bitmaps);
    if (counts) cudaFree(counts);
    if (nnz) cudaFree(nnz);
    if (ql) cudaFree(ql);
    if (qoff) cudaFree(qoff);
    for (auto *pp : packed)
      if (pp) cudaFree(pp);
    if (nnz_host) cudaFreeHost(nnz_host);
    if (ql_host) cudaFreeHost(ql_host);
    if (qoff_host) cudaFreeHost(qoff_host);
    for (auto *pp : packed_host)
      if (pp) cudaFreeHost(pp);
    for (auto e : ev) cudaEventDestroy(e);
    if (up) cudaStreamDestroy(up);
    if (compute) cudaStreamDestroy(compute);
    if (copy) cudaStreamDestroy(copy);
  }
};
void destroy_host_batch(HostBatchBuffers *b) { delete b; }

// Pinned host memory of at least `count` elements (grown, contents dropped).
template <class T>
static void ensure_host(T *&p, size_t &cap, size_t count) {
  if (cap >= count) return;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  if (cudaHostAlloc(reinterpret_cast<void **>(&p), std::max<size_t>(count, 1) * sizeof(T), 0) != cudaSuccess) {
    cudaGetLastError();
    throw Error(RTS_ERR_NOMEM, "pinned host allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  cap = count;
}

template <class T>
static void ensure(T *&p, size_t &cap, size_t count) {
  if (cap >= count) return;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    throw Error(RTS_ERR_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  cap = count;
}
}  // namespace rts

// Host columns in, host bitmaps out: upload, batched passes, download, with
// the download of each chunk of queries overlapping the next chunk's pass.
extern "C" rts_status rts_scan_batch_host(rts_ctx *ctx, const uint32_t *const *host_cols, int32_t ncols,
                                          uint64_t nrows, const rts_term *terms, const int32_t *offsets, int32_t nq,
                                          uint32_t *host_bitmaps, uint64_t stride_words, uint64_t *host_counts) {
  rts::Range nvtx_range_("rts_scan_batch_host");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!host_cols || ncols < 1 || nrows == 0) throw rts::Error(RTS_ERR_ARG, "need host columns");
    for (int c = 0; c < ncols; c++)
      if (!host_cols[c]) throw rts::Error(RTS_ERR_ARG, "null column pointer");
    if (nq < 0 || (nq > 0 && (!offsets || !host_bitmaps || !host_counts)))
      throw rts::Error(RTS_ERR_ARG, "bad batch arguments");
    const uint64_t words = rts::words_for(nrows);
    if (stride_words < words) throw rts::Error(RTS_ERR_ARG, "stride_words smaller than a bitmap");
    rts::DeviceGuard device_guard(ctx->device);
    if (!ctx->host_batch) ctx->host_batch = new rts::HostBatchBuffers();
    rts::HostBatchBuffers &H = *ctx->host_batch;
    if (!H.up) RTS_CUDA(cudaStreamCreateWithFlags(&H.up, cudaStreamNonBlocking));
    if (!H.compute) RTS_CUDA(cudaStreamCreateWithFlags(&H.compute, cudaStreamNonBlocking));
    if (!H.copy) RTS_CUDA(cudaStreamCreateWithFlags(&H.copy, cudaStreamNonBlocking));
    const uint64_t cstride = (nrows + 3) / 4 * 4;
    rts::ensure(H.cols, H.cols_cap, (size_t)cstride * ncols);
    rts::ensure(H.bitmaps, H.bm_cap, (size_t)std::max(nq, 1) * stride_words);
    rts::ensure(H.counts, H.cnt_cap, (size_t)std::max(nq, 1));
    // The batch kernels read the uploaded columns through the context.
    std::vector<const uint32_t *> saved_cols = ctx->cols;
    const uint64_t saved_n = ctx->nrows;
    ctx->cols.clear();
    for (int c = 0; c < ncols; c++) ctx->cols.push_back(H.cols + cstride * c);
    ctx->nrows = nrows;
    // On every way out: no copy from the caller's buffers is left in flight,
    // and the context's own columns are back.
    struct Restore {
      rts_ctx *c;
      std::vector<const uint32_t *> cols;
      uint64_t n;
      rts::HostBatchBuffers *h;
      ~Restore() {
        cudaStreamSynchronize(h->up);
        cudaStreamSynchronize(h->compute);
        cudaStreamSynchronize(h->copy);
        c->cols = cols;
        c->nrows = n;
      }
    } restore{ctx, saved_cols, saved_n, &H};
    // Row-chunked pipeline over three streams: the upload of chunk r+1 and
    // the download of chunk r-1's words of every bitmap (one 2D copy) run
    // while chunk r is scanned, so the column upload hides under the bitmap
    // download.  Chunks are multiples of 4096 rows (the largest kernel block).
    // Chunks of about 2^22 rows (at most 32): the first download starts
    // after one chunk's upload and scan.  Each chunk's upload is queued with
    // its scan (queueing every upload first measured 21 ms slower per 1e8 x 4
    // call: the downloads then share the link with 1.6 GB of uploads).
    const uint64_t want_chunks = std::max<uint64_t>(1, std::min<uint64_t>(32, nrows >> 22));
    const uint64_t chunk_rows = ((nrows + want_chunks - 1) / want_chunks + 4095) / 4096 * 4096;
    const int nchunks = (int)((nrows + chunk_rows - 1) / chunk_rows);
    // events per chunk: upload, scan, counts on the host, pack, packed words on the host
    const int kEv = 5;
    while ((int)H.ev.size() < kEv * nchunks + 1) {
      cudaEvent_t e;
      RTS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      H.ev.push_back(e);
    }
    auto ev = [&](int r, int k) { return H.ev[kEv * r + k]; };
    std::vector<rts::NormQuery> norm = rts::normalize_all(ctx, terms, offsets, nq);
    std::vector<int> inside, outside;
    for (int q = 0; q < nq; q++) (rts::runs_in_kernel(norm[q]) ? inside : outside).push_back(q);
    std::vector<char> is_outside(std::max(nq, 1), 0);
    for (int q : outside) is_outside[q] = 1;
    if (nq > 0) RTS_CUDA(cudaMemsetAsync(H.counts, 0, (size_t)nq * 8, H.compute));
    H.last_h2d = (uint64_t)nrows * 4 * ncols;  // and below: the plan, the packed-query lists
    H.last_d2h = (uint64_t)nq * 8;             // and below: bitmaps, packed chunks, nonzero-word counts
    rts::BatchPlan plan;
    const uint32_t *dev_blob = nullptr;
    cudaEvent_t blob_done = nullptr;
    void *pre = nullptr;
    size_t pre_bytes = 0;
    if (!inside.empty()) {
      plan = rts::build_plan(ctx, norm, inside, nullptr, ctx->batch_cfg.table_budget, true);
      dev_blob = rts::upload_plan(ctx, plan, H.compute, &blob_done);
      H.last_h2d += plan.blob.size() * 4;
      pre_bytes = rts::plan_pre_bytes(plan, chunk_rows);
      pre = rts::context_pre_scratch(ctx, pre_bytes, H.compute);
    }
    // Sparse transfer (sparse_d2h.cuh) when a chunk holds enough words per
    // query; a packed query takes at most kPackNum / kPackDen of the chunk's
    // words.
    const uint64_t cw_max = chunk_rows / 32;
    const bool sparse = nq > 0 && !inside.empty() && cw_max >= rts::kSparseMinWords;
    // packed words per chunk: every packed query's, up to kSparseMaxWords (a query
    // that would pass it is sent whole)
    const uint64_t max_packed =
        sparse ? std::min<uint64_t>((uint64_t)nq * (cw_max * rts::kPackNum / rts::kPackDen), rts::kSparseMaxWords)
               : 0;
    if (sparse) {
      rts::ensure(H.nnz, H.nnz_cap, (size_t)nq * nchunks);
      rts::ensure_host(H.nnz_host, H.nnz_host_cap, (size_t)nq * nchunks);
      rts::ensure(H.ql, H.ql_cap, (size_t)nq * nchunks);
      rts::ensure(H.qoff, H.qoff_cap, (size_t)nq * nchunks);
      rts::ensure_host(H.ql_host, H.ql_host_cap, (size_t)nq * nchunks);
      rts::ensure_host(H.qoff_host, H.qoff_host_cap, (size_t)nq * nchunks);
      for (int i = 0; i < 2; i++) rts::ensure(H.packed[i], H.packed_cap[i], (size_t)max_packed);
      for (int i = 0; i < 3; i++) rts::ensure_host(H.packed_host[i], H.packed_host_cap[i], (size_t)max_packed);
    }
    // Host threads that expand packed queries (declared after the buffers'
    // owner, so that they are joined on every way out before the streams
    // are drained; they only wait for events already recorded).
    rts::SlotGate gate;
    std::unique_ptr<rts::TaskPool> pool;
    if (sparse) {
      const unsigned hw = std::thread::hardware_concurrency();
      pool.reset(new rts::TaskPool((int)std::max(1u, std::min(8u, hw ? hw / 2 : 4u))));
    }
    // Finish chunk r once its counts are on the host: the dense queries'
    // words leave as one 2D copy per run of consecutive dense queries, the
    // packed ones as masks and values expanded by the pool.
    auto finish = [&](int r) {
      const uint64_t r0 = (uint64_t)r * chunk_rows, r1 = std::min<uint64_t>(nrows, r0 + chunk_rows);
      const uint64_t w0 = r0 / 32, w1 = r1 == nrows ? words : r1 / 32, cw = w1 - w0;
      std::vector<int> packed;
      uint64_t total = 0;
      const bool try_pack = sparse && cw >= rts::kSparseMinWords;
      if (try_pack) RTS_CUDA(cudaEventSynchronize(ev(r, 2)));
      int32_t *qlh = H.ql_host + (size_t)nq * r;
      uint64_t *qoh = H.qoff_host + (size_t)nq * r;
      // a packed query's words: its mask (one bit per word) and its nonzero
      // words; it is packed when they take at most kPackNum / kPackDen of the
      // chunk and fit the staging slot
      auto packed_words = [&](int i) { return (cw + 31) / 32 + H.nnz_host[(size_t)nq * r + i]; };
      auto packs = [&](int i) {
        return try_pack && packed_words(i) * rts::kPackDen <= cw * rts::kPackNum &&
               total + packed_words(i) <= max_packed;
      };
      int q = 0;
      while (q < nq) {
        if (is_outside[q]) {
          q++;
          continue;
        }
        if (packs(q)) {
          const uint64_t c = packed_words(q);
          qlh[packed.size()] = q;
          qoh[packed.size()] = total;
          packed.push_back(q);
          total += c;
          q++;
          continue;
        }
        int qb = q + 1;  // a run of dense queries
        while (qb < nq && !is_outside[qb] && !packs(qb)) qb++;
        RTS_CUDA(cudaMemcpy2DAsync(host_bitmaps + (uint64_t)q * stride_words + w0, stride_words * 4,
                                   H.bitmaps + (uint64_t)q * stride_words + w0, stride_words * 4, cw * 4,
                                   (size_t)(qb - q), cudaMemcpyDeviceToHost, H.copy));
        H.last_d2h += cw * 4 * (uint64_t)(qb - q);
        q = qb;
      }
      if (packed.empty()) return;
      const int np = (int)packed.size();
      const int ds = r % 2, hs = r % 3;
      gate.wait_free(hs);
      int32_t *qld = H.ql + (size_t)nq * r;
      uint64_t *qod = H.qoff + (size_t)nq * r;
      RTS_CUDA(cudaMemcpyAsync(qld, qlh, np * sizeof(int32_t), cudaMemcpyHostToDevice, H.compute));
      RTS_CUDA(cudaMemcpyAsync(qod, qoh, np * sizeof(uint64_t), cudaMemcpyHostToDevice, H.compute));
      H.last_h2d += (uint64_t)np * (sizeof(int32_t) + sizeof(uint64_t));
      if (r >= 2) RTS_CUDA(cudaStreamWaitEvent(H.compute, ev(r - 2, 4), 0));  // the device slot's last copy
      rts::pack_kernel<<<np, rts::kPackThreads, 0, H.compute>>>(H.bitmaps, stride_words, w0, w1, qld, qod,
                                                               H.packed[ds]);
      ctx->launches++;
      RTS_CUDA(cudaEventRecord(ev(r, 3), H.compute));
      RTS_CUDA(cudaStreamWaitEvent(H.copy, ev(r, 3), 0));
      if (total)
        RTS_CUDA(cudaMemcpyAsync(H.packed_host[hs], H.packed[ds], total * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 H.copy));
      H.last_d2h += total * sizeof(uint32_t);
      RTS_CUDA(cudaEventRecord(ev(r, 4), H.copy));
      const int tasks = std::min(np, pool->size());
      gate.add(hs, tasks);
      cudaEvent_t e = ev(r, 4);
      const uint32_t *ph = H.packed_host[hs];
      const int dev = ctx->device;
      for (int t = 0; t < tasks; t++)
        pool->post([=, &gate] {
          cudaSetDevice(dev);
          cudaEventSynchronize(e);
          for (int j = t; j < np; j += tasks)
            rts::expand_mask(host_bitmaps + (uint64_t)qlh[j] * stride_words + w0, cw, ph + qoh[j]);
          gate.done(hs);
        });
    };
    for (int r = 0; r < nchunks; r++) {
      const uint64_t r0 = (uint64_t)r * chunk_rows, r1 = std::min<uint64_t>(nrows, r0 + chunk_rows);
      for (int c = 0; c < ncols; c++)
        RTS_CUDA(cudaMemcpyAsync(H.cols + cstride * c + r0, host_cols[c] + r0, (r1 - r0) * 4,
                                 cudaMemcpyHostToDevice, H.up));
      RTS_CUDA(cudaEventRecord(ev(r, 0), H.up));
      RTS_CUDA(cudaStreamWaitEvent(H.compute, ev(r, 0), 0));
      if (!inside.empty())
        ctx->launches += rts::launch_plan(ctx, plan, dev_blob, H.bitmaps, stride_words, H.counts, r0, r1, pre,
                                          pre_bytes, H.compute);
      RTS_CUDA(cudaEventRecord(ev(r, 1), H.compute));
      RTS_CUDA(cudaStreamWaitEvent(H.copy, ev(r, 1), 0));
      const uint64_t w0 = r0 / 32, w1 = r1 == nrows ? words : r1 / 32;
      if (sparse && w1 - w0 >= rts::kSparseMinWords) {
        rts::nnz_kernel<<<nq, rts::kSparseThreads, 0, H.compute>>>(H.bitmaps, stride_words, w0, w1,
                                                                   H.nnz + (size_t)nq * r);
        ctx->launches++;
        RTS_CUDA(cudaMemcpyAsync(H.nnz_host + (size_t)nq * r, H.nnz + (size_t)nq * r, (size_t)nq * 4,
                                 cudaMemcpyDeviceToHost, H.compute));
        H.last_d2h += (uint64_t)nq * 4;
        RTS_CUDA(cudaEventRecord(ev(r, 2), H.compute));
      }
      if (r >= 1) finish(r - 1);  // while chunk r runs
    }
    if (nq > 0) finish(nchunks - 1);
    // Queries outside the batch kernels read the whole table: after the last
    // upload (ordered on the compute stream), then their whole bitmaps.
    if (!outside.empty()) {
      ctx->launches += rts::launch_outside(ctx, norm, outside, nullptr, H.bitmaps, stride_words, H.counts, H.compute);
      RTS_CUDA(cudaEventRecord(H.ev[kEv * nchunks], H.compute));
      RTS_CUDA(cudaStreamWaitEvent(H.copy, H.ev[kEv * nchunks], 0));
      for (int q : outside) {
        RTS_CUDA(cudaMemcpyAsync(host_bitmaps + (uint64_t)q * stride_words, H.bitmaps + (uint64_t)q * stride_words,
                                 words * 4, cudaMemcpyDeviceToHost, H.copy));
        H.last_d2h += words * 4;
      }
    }
    if (blob_done) RTS_CUDA(cudaEventRecord(blob_done, H.compute));
    if (pre) rts::context_pre_done(ctx, H.compute);
    RTS_CUDA(cudaGetLastError());
    if (nq > 0) {
      RTS_CUDA(cudaEventRecord(H.ev[kEv * nchunks], H.compute));
      RTS_CUDA(cudaStreamWaitEvent(H.copy, H.ev[kEv * nchunks], 0));
      RTS_CUDA(cudaMemcpyAsync(host_counts, H.counts, (size_t)nq * 8, cudaMemcpyDeviceToHost, H.copy));
    }
    RTS_CUDA(cudaStreamSynchronize(H.copy));
    RTS_CUDA(cudaStreamSynchronize(H.compute));
    RTS_CUDA(cudaStreamSynchronize(H.up));
    pool.reset();  // every packed query expanded
    return RTS_OK;
  } catch (const rts::Error &e) {
    ctx->err = e.what();
    return rts::set_thread_error(e.code, e.what());
  } catch (const std::exception &e) {
    ctx->err = e.what();
    return rts::set_thread_error(RTS_ERR_NOMEM, e.what());
  }
}

extern "C" rts_status rts_host_transfer_bytes(const rts_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes) {
  if (!ctx || !h2d_bytes || !d2h_bytes) return rts::set_thread_error(RTS_ERR_ARG, "null argument");
  const rts::HostBatchBuffers *H = ctx->host_batch;
  *h2d_bytes = H ? H->last_h2d : 0;
  *d2h_bytes = H ? H->last_d2h : 0;
  return RTS_OK;
}

extern "C" rts_status rts_scan_batch_async(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int32_t nq,
                                           uint32_t *dev_bitmaps, uint64_t stride_words, uint64_t *dev_counts,
                                           void *stream) {
  rts::Range nvtx_range_("rts_scan_batch_async");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (ctx->cols.empty()) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (nq < 0 || (nq > 0 && (!offsets || !dev_bitmaps || !dev_counts)))
      throw rts::Error(RTS_ERR_ARG, "bad batch arguments");
    if (stride_words < rts::words_for(ctx->nrows)) throw rts::Error(RTS_ERR_ARG, "stride_words smaller than a bitmap");
    if (nq == 0) return RTS_OK;
    rts::DeviceGuard device_guard(ctx->device);
    rts::batch_scan(ctx, terms, offsets, nq, dev_bitmaps, stride_words,
                    reinterpret_cast<unsigned long long *>(dev_counts), (cudaStream_t)stream,
                    ctx->batch_cfg.table_budget);
    return RTS_OK;
  } catch (const rts::Error &e) {
    ctx->err = e.what();
    return rts::set_thread_error(e.code, e.what());
  } catch (const std::exception &e) {
    ctx->err = e.what();
    return rts::set_thread_error(RTS_ERR_NOMEM, e.what());
  }
}
