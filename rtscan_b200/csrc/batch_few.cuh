// Batched kernel for passes of few queries: at most 32 slots, and the
// planner sends passes of up to kFewMaxQueries (included by batch.cu inside
// its anonymous namespace; uses kFull and kMaxCols from there).
//
// With few queries the table-driven kernel's per-row work (interval
// positions, table loads, bit transposes) is shared by too few queries to
// pay off, so each row is tested against each term directly: a lane holds
// one row's column values, and one ballot per query and 32 rows gives a
// result word.  A warp covers a 1024-row tile in chunks of Q queries whose
// terms it reads from the kernel parameters; lane t keeps the ballot of
// rows 32t .. 32t+31 of each query of the chunk, so a query's 32 words
// leave as one 128-byte line straight from registers.  Q is a template
// parameter chosen per pass (few_chunk()): the pass's own count for one or
// two queries, else the most that the column count leaves room for.  One
// chunk size per kernel: a kernel holding several ran its main chunk
// 5-9 % slower on B200.
constexpr int kFewSlots = 32;
// Passes of at most this many queries run term by term.  On one 2^23-row
// segment of 4 columns the term-by-term kernel takes about 134 us at 16
// queries and 185 us at 24, a 128-slot table pass 160-165 us at any count.
constexpr int kFewMaxQueries = 20;
constexpr int kFewWarps = 8;

struct FewPass {
  const uint32_t *col[kMaxCols];
  uint2 term[kFewSlots][kMaxCols];  // (lo, hi - lo) of slot s on pass column c; (0, 2^32 - 1) if unconstrained
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

// Most queries per chunk over ncols columns.  Each chunk reads the tile's
// columns once (from L1/L2 after the first), so fewer columns leave room
// for more queries per chunk.
constexpr int few_chunk_max(int ncols) { return ncols <= 2 ? 8 : ncols <= 4 ? 4 : 2; }
// Queries per chunk for a pass of nq queries over ncols columns.
inline int few_chunk(int nq, int ncols) {
  const int q = few_chunk_max(ncols);
  return nq < q ? (nq <= 1 ? 1 : nq <= 2 ? 2 : q) : q;
}

template <int C, int Q>
__global__ void __launch_bounds__(kFewWarps * 32, 4) batch_few_kernel(const __grid_constant__ FewPass p) {
  __shared__ unsigned long long cnt[kFewSlots];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < kFewSlots) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int nq = p.nq;
  const uint64_t gw = (uint64_t)blockIdx.x * kFewWarps + warp, nw = (uint64_t)gridDim.x * kFewWarps;
  unsigned long long mine = 0;  // lane j: matches of query j in this warp's tiles
  for (uint64_t tile = p.tile_begin + gw; tile < p.ntiles; tile += nw) {
    const uint64_t row0 = tile * 1024, word = tile * 32 + lane;
    for (int j0 = 0; j0 < nq; j0 += Q) {
      // slots past nq (the last chunk's) hold always-true terms; their
      // results are neither stored nor counted
      uint2 tm[Q][C];
#pragma unroll
      for (int jj = 0; jj < Q; jj++)
#pragma unroll
        for (int c = 0; c < C; c++) tm[jj][c] = p.term[(j0 + jj) & (kFewSlots - 1)][c];
      uint32_t r[Q];  // lane t: the ballot of rows row0 + 32t .. row0 + 32t + 31
#pragma unroll
      for (int jj = 0; jj < Q; jj++) r[jj] = 0;
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
        const bool own = lane == t;
#pragma unroll
        for (int jj = 0; jj < Q; jj++) {
          bool pass = in;
#pragma unroll
          for (int c = 0; c < C; c++) pass = pass && (v[c] - tm[jj][c].x <= tm[jj][c].y);
          const uint32_t b = __ballot_sync(kFull, pass);
          r[jj] = own ? b : r[jj];
        }
      }
#pragma unroll
      for (int jj = 0; jj < Q; jj++) {
        const int j = j0 + jj;
        if (j < nq) {
          const uint32_t w = __brev(r[jj]);  // row 32t + i -> bit 31 - i
          const int32_t sq = p.slot_query[j];
          if (sq >= 0 && word < p.words) p.out[(uint64_t)sq * p.stride_words + word] = w;
          const uint32_t total = __reduce_add_sync(kFull, (uint32_t)__popc(w));
          if (lane == j) mine += total;
        }
      }
    }
  }
  if (lane < nq && mine) atomicAdd(&cnt[lane], mine);
  __syncthreads();
  if (threadIdx.x < nq && cnt[threadIdx.x] && p.slot_query[threadIdx.x] >= 0)
    atomicAdd(p.counts + p.slot_query[threadIdx.x], cnt[threadIdx.x]);
}

template <int C>
void launch_few(const FewPass &fp, int grid, cudaStream_t s) {
  constexpr int Q = few_chunk_max(C);
  switch (few_chunk(fp.nq, C)) {
    case 1: batch_few_kernel<C, 1><<<grid, kFewWarps * 32, 0, s>>>(fp); break;
    case 2: batch_few_kernel<C, 2><<<grid, kFewWarps * 32, 0, s>>>(fp); break;
    default: batch_few_kernel<C, Q><<<grid, kFewWarps * 32, 0, s>>>(fp); break;
  }
}
