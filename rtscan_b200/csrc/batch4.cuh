// Batched kernel with table-driven passes of up to 512 queries (included by
// batch.cu inside its anonymous namespace; uses BatchPass, position_fast(),
// position() and kFull from there).
//
// A pass has GV groups of 32 query slots (GV = 16, 8 or 4: 512, 256 or 128
// slots; the planner picks the smallest that holds the pass), and its
// tables hold GV words per interval position.  A CTA of W warps (16, or 8
// so that two CTAs can share an SM when the tables are small) works on
// blocks of W x 32 x 32 / GV rows (1024, 2048, 4096 for 16 warps): tiles of
// 32 rows, 32 / GV tiles per warp, and all slots of the pass at once:
//   1. every thread finds the interval positions of 32 / GV rows (one per
//      column) and writes their table word offsets to shared memory, while
//      the previous block's result words are stored;
//   2. lane (tile t = (32 / GV) * warp + lane / GV, group g = lane % GV) ANDs
//      the table words of its tile's 32 rows for group g (one shared-memory
//      load per row and column), then bit-transposes the 32 masks in
//      registers so that word j holds query 32g+j's 32 row bits, MSB-first,
//      and writes the 32 words to a shared-memory stage laid out
//      [query][tiles of the block] with word index t ^ ((32 / GV) * g),
//      which puts the 32 lanes of a warp in 32 different banks;
//   3. each warp stores 32 * GV / W queries' rows of the stage: a query's
//      words for the block (128 bytes per 1024 rows) leave as 16-byte stores
//      from 128 / GV lanes, whole 128-byte lines.
// No cross-lane exchange is needed, and positions are shared by all queries
// of the pass.  16-warp passes over up to four columns run step 2 with
// wide lanes (16 rows x two groups, 8-byte table loads, 16-bit stage
// halves; see the kernel): their loads per mask bit are halved, which
// measured 2.9 % faster per 1024-query step (passes reading shared
// positions), 1.8 % faster for 400- and 512-query batches and 20-22 %
// faster for 64- and 128-query ones.  For 512- and 256-slot passes over up
// to 4 columns, and every pass reading shared positions, step 1 for the
// next block runs inside step 2 (see the kernel).
template <int GV, int W>
struct V4Shape {
  static_assert(GV == 16 || GV == 8 || GV == 4, "512-, 256- or 128-slot passes");
  static_assert(W == 16 || W == 8, "8 or 16 warps per CTA");
  static constexpr int kThreads = W * 32;
  static constexpr int kTPW = 32 / GV;               // tiles per warp
  static constexpr int kTiles = W * kTPW;            // tiles per block = words per query per block
  static constexpr int kRows = kTiles * 32;          // rows per block
  static constexpr int kSlots = 32 * GV;
  static constexpr int kStage = kSlots * kTiles;     // stage words: 1024 * W
  static constexpr int kRPT = kRows / kThreads;      // rows per thread in step 1
  static constexpr int kLPQ = kTiles / 4;            // lanes per query row in step 3 (16-byte chunks)
  static constexpr int kQPI = 32 / kLPQ;             // queries per store instruction
  static constexpr int kQPW = kSlots / W;            // queries each warp stores in step 3
  static constexpr int kIters = kQPW / kQPI;         // store instructions per warp and block (8)
  // Stage word-index XOR of group g: kTPW * g, kept below kTiles (with 16
  // warps it always is; 512 slots on 8 warps fold it, and their stage
  // writes then meet two to a bank)
  static __device__ __forceinline__ int swizzle(int g) { return (kTPW * g) & (kTiles - 1); }
  static_assert(kIters == 8, "eight store instructions per warp");
};

// Per row and column the position buffer holds the word offset of the row's
// table entry (table start + position * GV), to which a lane adds its group:
// 32-bit entries for up to 4 columns, 16-bit ones for 8 (a pass blob is
// under 2^16 words), one padding row per tile.
template <int CMAX>
using V4Pos = typename std::conditional<(CMAX <= 4), uint32_t, uint16_t>::type;
// (16 warps over up to four columns: one padding row per 16, for the wide
// lanes of batch4_kernel)
template <int CMAX, int GV, int W>
constexpr int kV4PosBytes =
    (V4Shape<GV, W>::kRows + ((W == 16 && CMAX == 4) ? V4Shape<GV, W>::kRows / 16 : V4Shape<GV, W>::kTiles)) *
    CMAX * (int)sizeof(V4Pos<CMAX>);

// Exchange the bits of a under mask M << S with the bits of b under M (a
// delta swap: the XOR of the two bit sets applied to both; measured faster
// here than two shift-and-select results).
template <int S, uint32_t M>
__device__ __forceinline__ void swap_bits(uint32_t &a, uint32_t &b) {
  const uint32_t t = ((a >> S) ^ b) & M;
  b ^= t;
  a ^= t << S;
}

// 32x32 bit transpose in registers: on return bit j of x[i] is the input's
// bit i of x[j].  Each stage exchanges one bit of the row index with the
// same bit of the column index, so the stages commute: three delta swaps
// (1-, 2-, 4-bit blocks) and then two byte-permute stages (8-, 16-bit), the
// order measured fastest.
__device__ __forceinline__ void transpose32(uint32_t (&x)[32]) {
#pragma unroll
  for (int i = 0; i < 32; i += 2) swap_bits<1, 0x55555555u>(x[i], x[i + 1]);
#pragma unroll
  for (int base = 0; base < 32; base += 4) {
#pragma unroll
    for (int i = base; i < base + 2; i++) swap_bits<2, 0x33333333u>(x[i], x[i + 2]);
  }
#pragma unroll
  for (int base = 0; base < 32; base += 8) {
#pragma unroll
    for (int i = base; i < base + 4; i++) swap_bits<4, 0x0F0F0F0Fu>(x[i], x[i + 4]);
  }
#pragma unroll
  for (int base = 0; base < 32; base += 16) {
#pragma unroll
    for (int i = base; i < base + 8; i++) {
      const uint32_t a = x[i], b = x[i + 8];
      x[i] = __byte_perm(a, b, 0x6240);      // 8x8 blocks: bytes 1<->0 and 3<->2
      x[i + 8] = __byte_perm(a, b, 0x7351);
    }
  }
#pragma unroll
  for (int i = 0; i < 16; i++) {  // the off-diagonal 16x16 blocks
    const uint32_t a = x[i], b = x[i + 16];
    x[i] = __byte_perm(a, b, 0x5410);       // low halves: a.lo | b.lo << 16
    x[i + 16] = __byte_perm(a, b, 0x7632);  // high halves: a.hi | b.hi << 16
  }
}

// Two 16x16 bit transposes at once, one in each 16-bit half of 16 words: on
// return bit j of x[i] is the input's bit i of x[j], and bit 16 + j of x[i]
// the input's bit 16 + i of x[j] (i, j < 16).  The stages of transpose32
// without its 16-bit one.
__device__ __forceinline__ void transpose16x2(uint32_t (&x)[16]) {
#pragma unroll
  for (int i = 0; i < 16; i += 2) swap_bits<1, 0x55555555u>(x[i], x[i + 1]);
#pragma unroll
  for (int base = 0; base < 16; base += 4) {
#pragma unroll
    for (int i = base; i < base + 2; i++) swap_bits<2, 0x33333333u>(x[i], x[i + 2]);
  }
#pragma unroll
  for (int base = 0; base < 16; base += 8) {
#pragma unroll
    for (int i = base; i < base + 4; i++) swap_bits<4, 0x0F0F0F0Fu>(x[i], x[i + 4]);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t a = x[i], b = x[i + 8];
    x[i] = __byte_perm(a, b, 0x6240);  // bytes 1 <-> 0 and 3 <-> 2 of the pair
    x[i + 8] = __byte_perm(a, b, 0x7351);
  }
}

// PRE: the batch's positions were found once for all its passes
// (pre_kernel in batch.cu), and this pass reads its rows' table word
// offsets (four uint16 per row) from p.pre instead of searching; only for
// the shapes that find positions a block ahead.
template <int CMAX, int GV, int W, bool PRE>
__global__ void __launch_bounds__(W * 32, 16 / W) batch4_kernel(const __grid_constant__ BatchPass p) {
  using S = V4Shape<GV, W>;
  constexpr int kV4Threads = S::kThreads;
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *blob = smem;
  uint32_t *stage = smem + ((p.blob_words + 3) & ~3u);
  V4Pos<CMAX> *posbuf = reinterpret_cast<V4Pos<CMAX> *>(stage + S::kStage);

  for (uint32_t i = threadIdx.x; i < p.blob_words; i += blockDim.x) blob[i] = __ldg(p.blob + i);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int C = p.ncols;
  const int32_t *slot_query = reinterpret_cast<const int32_t *>(blob + p.slot_off);
  // step-2 identity
  const int tile = S::kTPW * warp + lane / GV, g = lane % GV;
  // step-3 identity: queries warp * kQPW + it * kQPI + qq, 16-byte chunk
  // `chunk` of their row; the stage word-index XOR of query q's group is
  // kTPW * (q / 32), constant over the kQPI queries of one instruction
  const int qq = lane / S::kLPQ, chunk = lane % S::kLPQ;
  uint32_t cnt[S::kIters];
#pragma unroll
  for (int i = 0; i < S::kIters; i++) cnt[i] = 0;

  // For 512- and 256-slot passes over up to 4 columns (3-5 % faster for the
  // 256-slot shape, 4-10 % slower for the 128-slot one, whose 8 rows per
  // thread are too many to hold), positions are found one block ahead,
  // inside step 2: even warps before their masks, odd warps after, so
  // the dependent shared-memory loads of the boundary search overlap other
  // warps' mask arithmetic; the table word offsets wait in registers as
  // 16-bit pairs until the next step 1 writes them to shared memory, and the
  // column values are loaded one more block ahead.  Other shapes find the
  // positions of a block in its own step 1.
  constexpr bool kAhead = (GV == 16 || GV == 8 || PRE) && CMAX <= 4;
  static_assert(!PRE || (kAhead && CMAX == 4), "shared positions feed the 4-column look-ahead shapes");
  uint32_t val[S::kRPT][CMAX];                    // column values of this thread's rows (PRE: packed offsets)
  uint32_t offn[kAhead ? S::kRPT : 1][(CMAX + 1) / 2];  // their table word offsets, two per register
  auto load_values = [&](uint64_t b) {
#pragma unroll
    for (int h = 0; h < S::kRPT; h++) {
      const uint64_t row = b * S::kRows + threadIdx.x + h * kV4Threads;
      if (PRE) {  // the row's four offsets, two per word, as find_offsets packs them
        const uint2 w = row < p.nrows ? __ldg(p.pre + (row - p.pre_row0)) : make_uint2(0u, 0u);
        val[h][0] = w.x;
        val[h][1] = w.y;
      } else {
#pragma unroll
        for (int c = 0; c < CMAX; c++) val[h][c] = (c < C && row < p.nrows) ? __ldg(p.col[c] + row) : 0u;
      }
    }
  };
  // kAhead: latency hidden behind the masks, so the search with the fewest
  // instructions
  auto row_offsets = [&](uint64_t b, int h, uint32_t(&off)[CMAX]) {
    const bool in = b * S::kRows + threadIdx.x + h * kV4Threads < p.nrows;
    uint32_t pos[CMAX];
#pragma unroll
    for (int c = 0; c < CMAX; c++) pos[c] = (c < C && in) ? position(p, blob, c, val[h][c]) : 0u;
#pragma unroll
    for (int c = 0; c < CMAX; c++) off[c] = c < C ? p.tab_off[c] + pos[c] * GV : 0u;
  };
  // Wide pass (16 warps, up to four columns): a lane takes 16
  // rows and 64 slots (two groups) of step 2, with 8-byte table loads; see
  // step 2.  The position buffer then has a padding row per 16
  // rows, so that the four 16-row tiles of a warp read it in different banks.
  constexpr bool kWide = W == 16 && CMAX == 4;
  auto pos_row = [](int r) { return kWide ? r + (r >> 4) : r + (r >> 5); };
  auto put_row = [&](int h, const uint32_t(&off)[CMAX]) {
    const int r = threadIdx.x + h * kV4Threads;
    V4Pos<CMAX> *dst = posbuf + pos_row(r) * CMAX;
    if (CMAX <= 4) {
      *reinterpret_cast<uint4 *>(dst) = make_uint4(off[0], off[1 % CMAX], off[2 % CMAX], off[3 % CMAX]);
    } else {
#pragma unroll
      for (int c = 0; c < CMAX; c += 4)
        *reinterpret_cast<uint2 *>(dst + c) =
            make_uint2(off[c] | (off[(c + 1) % CMAX] << 16), off[(c + 2) % CMAX] | (off[(c + 3) % CMAX] << 16));
    }
  };
  // Other shapes: loop-free lookups for up to 16 (row, column) pairs at once
  // (1 % faster than 32 for 128-slot passes), so that their shared-memory
  // loads overlap, and their offsets to shared memory; then the full search for the few whose bucket is crowded, each
  // lane over its own misses only (a column value read again, from cache),
  // overwriting those entries.
  auto block_offsets = [&](uint64_t b) {
    constexpr int H = (16 / CMAX) < S::kRPT ? (16 / CMAX) : S::kRPT;  // rows per batch of lookups
#pragma unroll
    for (int h0 = 0; h0 < S::kRPT; h0 += H) {
      uint32_t pos[H][CMAX];
      uint32_t miss[CMAX];  // bit hh: the lookup of (row h0 + hh, column c) was not exact
#pragma unroll
      for (int c = 0; c < CMAX; c++) miss[c] = 0;
#pragma unroll
      for (int hh = 0; hh < H; hh++) {
        const bool in = b * S::kRows + threadIdx.x + (h0 + hh) * kV4Threads < p.nrows;
#pragma unroll
        for (int c = 0; c < CMAX; c++) {
          bool e = true;
          pos[hh][c] = (c < C && in) ? position_fast(p, blob, c, val[h0 + hh][c], e) : 0u;
          miss[c] |= (e ? 0u : 1u) << hh;
        }
      }
#pragma unroll
      for (int hh = 0; hh < H; hh++) {
        uint32_t off[CMAX];
#pragma unroll
        for (int c = 0; c < CMAX; c++) off[c] = c < C ? p.tab_off[c] + pos[hh][c] * GV : 0u;
        put_row(h0 + hh, off);
      }
#pragma unroll
      for (int c = 0; c < CMAX; c++) {
        uint32_t mc = miss[c];
        while (mc) {
          const int hh = __ffs(mc) - 1;
          mc &= mc - 1;
          const int r = threadIdx.x + (h0 + hh) * kV4Threads;
          const uint32_t x = __ldg(p.col[c] + b * S::kRows + r);
          posbuf[pos_row(r) * CMAX + c] = (V4Pos<CMAX>)(p.tab_off[c] + position(p, blob, c, x) * GV);
        }
      }
    }
  };
  auto find_offsets = [&](uint64_t b) {  // kAhead: into offn
#pragma unroll
    for (int h = 0; h < S::kRPT; h++) {
      if (PRE) {
        offn[h % (kAhead ? S::kRPT : 1)][0] = val[h][0];
        offn[h % (kAhead ? S::kRPT : 1)][1 % ((CMAX + 1) / 2)] = val[h][1];
      } else {
        uint32_t off[CMAX];
        row_offsets(b, h, off);
#pragma unroll
        for (int c = 0; c < CMAX; c += 2)
          offn[h % (kAhead ? S::kRPT : 1)][c / 2] = off[c] | (c + 1 < CMAX ? off[c + 1] << 16 : 0u);
      }
    }
  };
  auto put_offsets = [&]() {  // kAhead: from offn
#pragma unroll
    for (int h = 0; h < S::kRPT; h++) {
      uint32_t off[CMAX];
#pragma unroll
      for (int c = 0; c < CMAX; c++) {
        const uint32_t w = offn[h % (kAhead ? S::kRPT : 1)][c / 2];
        off[c] = (c & 1) ? w >> 16 : w & 0xFFFF;
      }
      put_row(h, off);
    }
  };

  const uint64_t nblocks = p.nblocks, step = gridDim.x;
  uint64_t blk = p.block_begin + blockIdx.x;
  uint64_t prev = ~0ull;  // block whose stage is waiting to be stored
  if (kAhead && blk < nblocks) {
    load_values(blk);
    find_offsets(blk);
    if (blk + step < nblocks) load_values(blk + step);
  }
  while (true) {
    // ---- step 1: offsets of block `blk` to shared memory, store of block `prev` ----
    if (blk < nblocks) {
      if (kAhead) {
        put_offsets();
      } else {
        load_values(blk);
        block_offsets(blk);
      }
    }
    if (prev != ~0ull) {
      const uint64_t word0 = prev * S::kTiles;
      const bool full = p.vec_store && word0 + S::kTiles <= p.words;
#pragma unroll
      for (int it = 0; it < S::kIters; it++) {
        const int q = warp * S::kQPW + it * S::kQPI + qq;
        const int sw = S::swizzle((warp * S::kQPW + it * S::kQPI) >> 5);
        const int pchunk = chunk ^ (sw >> 2);  // physical chunk of logical chunk `chunk`
        const int32_t sq = slot_query[q];
        uint4 v = *reinterpret_cast<const uint4 *>(stage + q * S::kTiles + pchunk * 4);
        if (sw & 2) v = make_uint4(v.z, v.w, v.x, v.y);  // words k and k^2 swapped inside a chunk
        cnt[it] += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
        if (sq >= 0) {
          uint32_t *dst = p.out + (uint64_t)sq * p.stride_words + word0 + chunk * 4;
          if (full) {
            *reinterpret_cast<uint4 *>(dst) = v;
          } else {
            const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; k++)
              if (word0 + chunk * 4 + k < p.words) dst[k] = w4[k];
          }
        }
      }
    }
    __syncthreads();
    if (blk >= nblocks) break;
    // ---- step 2: masks, transpose, stage of `blk` (and offsets of the next block) ----
    const uint64_t nxt = blk + step;
    auto ahead = [&]() {
      if (kAhead && nxt < nblocks) {
        find_offsets(nxt);
        if (nxt + step < nblocks) load_values(nxt + step);
      }
    };
    if (!(warp & 1)) ahead();
    if constexpr (kWide) {
      // Wide lanes: 16-row tile k = lane / (GV / 2) of the warp (rows
      // 16hh .. 16hh + 15 of the block's 32-row tile T = kTPW * warp +
      // k % kTPW, hh = k / kTPW) and groups 2gp, 2gp + 1 (gp = lane %
      // (GV / 2)): one 8-byte table load per row
      // and column serves both groups, half the loads per mask bit of the
      // 32-row, one-group lanes; the two 16 x 32 masks are transposed as
      // 16 x 16 blocks in 16-bit halves and written to the stage as 16-bit
      // halves of its words (rows 0-15 the high half).
      const int k = lane / (GV / 2), gp = lane % (GV / 2);
      const int T = S::kTPW * warp + (k % S::kTPW), hh = k / S::kTPW;
      const int row0 = 32 * T + 16 * hh;
      const char *tabg = reinterpret_cast<const char *>(blob + 2 * gp);
      uint32_t x0[16], x1[16];
#pragma unroll
      for (int r = 0; r < 16; r++) {
        const uint4 pv = *reinterpret_cast<const uint4 *>(posbuf + pos_row(row0 + r) * CMAX);
        const uint32_t off[4] = {pv.x, pv.y, pv.z, pv.w};
        uint32_t a0 = 0xFFFFFFFFu, a1 = 0xFFFFFFFFu;
#pragma unroll
        for (int c = 0; c < 4; c++)
          if (c < C) {
            const uint2 t = *reinterpret_cast<const uint2 *>(tabg + off[c] * p.word_bytes);
            a0 &= t.x;
            a1 &= t.y;
          }
        x0[15 - r] = a0;  // reversed: after the transpose row 0 is bit 15 of a half
        x1[15 - r] = a1;
      }
      transpose16x2(x0);
      transpose16x2(x1);
      const uint64_t tile_row0 = blk * S::kRows + (uint64_t)row0;
      if (tile_row0 + 16 > p.nrows) {
        const uint64_t valid = tile_row0 < p.nrows ? p.nrows - tile_row0 : 0;
        const uint32_t v16 = valid >= 16 ? 0xFFFFu : (0xFFFFu << (16 - valid)) & 0xFFFFu;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          x0[j] &= v16 | v16 << 16;
          x1[j] &= v16 | v16 << 16;
        }
      }
      // x[i]: slot 32 gq + i in the low half, 32 gq + 16 + i in the high half
      uint16_t *st16 = reinterpret_cast<uint16_t *>(stage);
      const int half = hh ? 0 : 1;  // 16-bit index in the word (little-endian)
      auto put_group = [&](const uint32_t(&x)[16], int gq) {
        const int col = T ^ S::swizzle(gq);
#pragma unroll
        for (int i = 0; i < 16; i++) {
          st16[((32 * gq + i) * S::kTiles + col) * 2 + half] = (uint16_t)(x[i] & 0xFFFFu);
          st16[((32 * gq + 16 + i) * S::kTiles + col) * 2 + half] = (uint16_t)(x[i] >> 16);
        }
      };
      put_group(x0, 2 * gp);
      put_group(x1, 2 * gp + 1);
    } else {
      const uint64_t tile_row0 = blk * S::kRows + (uint64_t)tile * 32;
      const uint32_t *tabg = blob + g;
      uint32_t acc[32];
#pragma unroll
      for (int r = 0; r < 32; r++) {
        const int row = tile * 32 + r;
        const V4Pos<CMAX> *pr = posbuf + pos_row(row) * CMAX;
        uint32_t off[CMAX];
        if (CMAX <= 4) {
          const uint4 pv = *reinterpret_cast<const uint4 *>(pr);
          off[0] = pv.x;
          off[1 % CMAX] = pv.y;
          off[2 % CMAX] = pv.z;
          off[3 % CMAX] = pv.w;
        } else {
#pragma unroll
          for (int c = 0; c < CMAX; c += 4) {
            const uint2 pv = *reinterpret_cast<const uint2 *>(pr + c);
            off[c] = pv.x & 0xFFFF;
            off[(c + 1) % CMAX] = pv.x >> 16;
            off[(c + 2) % CMAX] = pv.y & 0xFFFF;
            off[(c + 3) % CMAX] = pv.y >> 16;
          }
        }
        uint32_t a = 0xFFFFFFFFu;
#pragma unroll
        for (int c = 0; c < CMAX; c++)
          if (c < C) {
            // 512 slots: the byte address as off * word_bytes + tabg with the
            // multiplier a run-time 4, which compiles to a multiply-add on the
            // FMA pipe instead of a shift-add on the busier integer ALU pipe
            // (2 % faster per pass on B200; the smaller shapes gain nothing)
            if (GV == 16)
              a &= *reinterpret_cast<const uint32_t *>(reinterpret_cast<const char *>(tabg) + off[c] * p.word_bytes);
            else
              a &= tabg[off[c]];
          }
        acc[31 - r] = a;  // reversed: after the transpose row 0 is the MSB
      }
      transpose32(acc);
      if (tile_row0 + 32 > p.nrows) {
        const uint64_t valid = tile_row0 < p.nrows ? p.nrows - tile_row0 : 0;
        const uint32_t vm = valid >= 32 ? 0xFFFFFFFFu : (valid ? ~(0xFFFFFFFFu >> valid) : 0u);
#pragma unroll
        for (int j = 0; j < 32; j++) acc[j] &= vm;
      }
      const int col = tile ^ S::swizzle(g);
#pragma unroll
      for (int j = 0; j < 32; j++) stage[(32 * g + j) * S::kTiles + col] = acc[j];
    }
    if (warp & 1) ahead();
    __syncthreads();
    prev = blk;
    blk = nxt;
  }
  // counts: the kLPQ lanes of a query row hold partial counts of that query
#pragma unroll
  for (int it = 0; it < S::kIters; it++) {
    uint32_t c = cnt[it];
#pragma unroll
    for (int o = 1; o < S::kLPQ; o <<= 1) c += __shfl_xor_sync(kFull, c, o);
    const int q = warp * S::kQPW + it * S::kQPI + qq;
    const int32_t sq = slot_query[q];
    if (chunk == 0 && sq >= 0 && c) atomicAdd(p.counts + sq, (unsigned long long)c);
  }
}
