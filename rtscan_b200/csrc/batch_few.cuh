// Batched kernel for passes of at most 32 queries (included by batch.cu
// inside its anonymous namespace; uses kFull and kMaxCols from there).
//
// With few queries the table-driven kernel's per-row work (interval
// positions, table loads, bit transposes) is shared by too few queries to
// pay off, so each row is tested against each term directly: a lane holds
// one row's column values, the terms of a chunk of queries sit in
// registers, and one ballot per query and 32 rows gives a result word.  A
// warp covers a 1024-row tile: the 32 ballots of a query are collected in
// shared memory and leave as one 128-byte line per query.  Cost per row and
// query is two instructions per pass column plus about three, against the
// columns' read traffic.
constexpr int kFewSlots = 32;
constexpr int kFewWarps = 8;

struct FewPass {
  const uint32_t *col[kMaxCols];
  uint2 term[kFewSlots][kMaxCols];  // (lo, hi - lo) of slot s on pass column c
  uint32_t colmask[kFewSlots];      // pass columns slot s constrains
  int32_t slot_query[kFewSlots];    // bitmap index of slot s, -1 when unused
  int nq;
  int ncols;
  uint32_t *out;
  uint64_t stride_words;
  unsigned long long *counts;
  uint64_t nrows;
  uint64_t words;
  uint64_t tile_begin;  // first 1024-row tile of the range
  uint64_t ntiles;      // end of the range, in tiles
};

template <int C>
__global__ void __launch_bounds__(kFewWarps * 32, 4) batch_few_kernel(const __grid_constant__ FewPass p) {
  // Queries go in chunks of QCH whose terms sit in registers (lo, hi - lo per
  // column; an unconstrained column has (0, 2^32 - 1), always true); the
  // chunk's 1024-row tile is read once per chunk (from L1/L2 after the first).
  constexpr int QCH = C <= 2 ? 8 : C <= 4 ? 4 : 2;
  __shared__ uint32_t stage[kFewWarps][kFewSlots][32];
  __shared__ uint2 term[kFewSlots][C];
  __shared__ unsigned long long cnt[kFewSlots];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < kFewSlots) {
    cnt[threadIdx.x] = 0;
    const bool used = threadIdx.x < p.nq;
#pragma unroll
    for (int c = 0; c < C; c++)
      term[threadIdx.x][c] = !used ? make_uint2(1u, 0u)  // never true: the slot is unused
                             : (p.colmask[threadIdx.x] >> c & 1) ? p.term[threadIdx.x][c]
                                                                  : make_uint2(0u, 0xFFFFFFFFu);
  }
  __syncthreads();
  const int nq = p.nq;
  const uint64_t gw = (uint64_t)blockIdx.x * kFewWarps + warp, nw = (uint64_t)gridDim.x * kFewWarps;
  for (uint64_t tile = p.tile_begin + gw; tile < p.ntiles; tile += nw) {
    const uint64_t row0 = tile * 1024;
    for (int j0 = 0; j0 < nq; j0 += QCH) {
      uint2 tm[QCH][C];
#pragma unroll
      for (int jj = 0; jj < QCH; jj++)
#pragma unroll
        for (int c = 0; c < C; c++) tm[jj][c] = term[(j0 + jj) & (kFewSlots - 1)][c];
      uint32_t nxt[C];
      auto load = [&](int t) {
        const uint64_t row = row0 + t * 32 + lane;
#pragma unroll
        for (int c = 0; c < C; c++) nxt[c] = row < p.nrows ? __ldg(p.col[c] + row) : 0u;
      };
      load(0);
      for (int t = 0; t < 32; t++) {
        uint32_t v[C];
#pragma unroll
        for (int c = 0; c < C; c++) v[c] = nxt[c];
        if (t + 1 < 32) load(t + 1);
        const bool in = row0 + t * 32 + lane < p.nrows;
#pragma unroll
        for (int jj = 0; jj < QCH; jj++) {
          bool pass = in;
#pragma unroll
          for (int c = 0; c < C; c++) pass = pass && (v[c] - tm[jj][c].x <= tm[jj][c].y);
          const uint32_t w = __brev(__ballot_sync(kFull, pass));  // row t*32 + i -> bit 31 - i
          if (lane == 0 && j0 + jj < nq) stage[warp][j0 + jj][t] = w;
        }
      }
    }
    __syncwarp();
    const uint64_t word = tile * 32 + lane;
    for (int j = 0; j < nq; j++) {
      const uint32_t w = stage[warp][j][lane];
      const int32_t sq = p.slot_query[j];
      if (sq >= 0 && word < p.words) p.out[(uint64_t)sq * p.stride_words + word] = w;
      const uint32_t total = __reduce_add_sync(kFull, (uint32_t)__popc(w));
      if (lane == 0 && total) atomicAdd(&cnt[j], (unsigned long long)total);
    }
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x < nq && cnt[threadIdx.x] && p.slot_query[threadIdx.x] >= 0)
    atomicAdd(p.counts + p.slot_query[threadIdx.x], cnt[threadIdx.x]);
}
