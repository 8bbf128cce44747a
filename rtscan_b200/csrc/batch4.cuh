// Batched kernel, 512-query passes (included by batch.cu inside its
// anonymous namespace; uses BatchPass, position() and kFull from there).
//
// A CTA of 16 warps works on blocks of 1024 rows (32 tiles of 32 rows) and
// all 512 query slots of the pass (16 groups of 32) at once:
//   1. every thread finds the interval positions of two rows (one per
//      column) and writes their table word offsets to shared memory, while
//      the previous block's result words are stored;
//   2. lane (tile t = 2*warp + lane/16, group g = lane%16) ANDs the table
//      words of its tile's 32 rows for group g (one shared-memory load per
//      row and column; the two tiles of a warp read two table rows), then
//      bit-transposes the 32 masks in registers so that word j holds query
//      32g+j's 32 row bits, MSB-first, and writes the 32 words to a
//      shared-memory stage laid out [query][32 words] with word index
//      tile ^ 2g, which puts the 32 lanes of a warp in 32 different banks;
//   3. each warp stores 32 queries' rows of the stage: a query's 32 words
//      (128 bytes, the block's 1024 rows) leave as eight 16-byte stores from
//      eight lanes, one full 128-byte line per query.
// No cross-lane exchange is needed, and positions are shared by all 512
// queries of the pass.  Step 1 for the next block runs inside step 2 (see
// the kernel), so one pair of barriers separates a block's steps.
constexpr int kV4Warps = 16;
constexpr int kV4Threads = kV4Warps * 32;
constexpr int kV4Groups = 16;
constexpr int kV4Slots = kV4Groups * 32;
constexpr int kV4Tiles = 32;  // tiles per block
constexpr int kV4Rows = kV4Tiles * 32;
constexpr int kV4StageWords = kV4Slots * kV4Tiles;  // 64 KB
// Per row and column the position buffer holds the word offset of the row's
// table entry (table start + position * 16), to which a lane adds its group:
// 32-bit entries for up to 4 columns, 16-bit ones for 8 (a pass blob is
// under 2^16 words), one padding row per tile.
template <int CMAX>
using V4Pos = typename std::conditional<(CMAX <= 4), uint32_t, uint16_t>::type;
template <int CMAX>
constexpr int kV4PosBytes = (kV4Rows + kV4Tiles) * CMAX * (int)sizeof(V4Pos<CMAX>);

// Exchange the bits of a under mask M << S with the bits of b under M:
// each result is one shift and one bitwise select.
template <int S, uint32_t M>
__device__ __forceinline__ void swap_bits(uint32_t &a, uint32_t &b) {
  const uint32_t na = (a & ~(M << S)) | ((b << S) & (M << S));
  const uint32_t nb = (b & ~M) | ((a >> S) & M);
  a = na;
  b = nb;
}

// 32x32 bit transpose in registers: on return bit j of x[i] is the input's
// bit i of x[j].  Two byte-permute stages (16, 8) and three delta swaps.
__device__ __forceinline__ void transpose32(uint32_t (&x)[32]) {
#pragma unroll
  for (int i = 0; i < 16; i++) {  // swap the off-diagonal 16x16 blocks
    const uint32_t a = x[i], b = x[i + 16];
    x[i] = __byte_perm(a, b, 0x5410);       // low halves: a.lo | b.lo << 16
    x[i + 16] = __byte_perm(a, b, 0x7632);  // high halves: a.hi | b.hi << 16
  }
#pragma unroll
  for (int base = 0; base < 32; base += 16) {
#pragma unroll
    for (int i = base; i < base + 8; i++) {  // 8x8 blocks: bytes 1<->0 and 3<->2
      const uint32_t a = x[i], b = x[i + 8];
      x[i] = __byte_perm(a, b, 0x6240);
      x[i + 8] = __byte_perm(a, b, 0x7351);
    }
  }
#pragma unroll
  for (int base = 0; base < 32; base += 8) {
#pragma unroll
    for (int i = base; i < base + 4; i++) swap_bits<4, 0x0F0F0F0Fu>(x[i], x[i + 4]);
  }
#pragma unroll
  for (int base = 0; base < 32; base += 4) {
#pragma unroll
    for (int i = base; i < base + 2; i++) swap_bits<2, 0x33333333u>(x[i], x[i + 2]);
  }
#pragma unroll
  for (int i = 0; i < 32; i += 2) swap_bits<1, 0x55555555u>(x[i], x[i + 1]);
}

template <int CMAX>
__global__ void __launch_bounds__(kV4Threads, 1) batch4_kernel(const __grid_constant__ BatchPass p) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *blob = smem;
  uint32_t *stage = smem + ((p.blob_words + 3) & ~3u);
  V4Pos<CMAX> *posbuf = reinterpret_cast<V4Pos<CMAX> *>(stage + kV4StageWords);

  for (uint32_t i = threadIdx.x; i < p.blob_words; i += blockDim.x) blob[i] = __ldg(p.blob + i);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int C = p.ncols;
  const int32_t *slot_query = reinterpret_cast<const int32_t *>(blob + p.slot_off);
  // compute-phase identity
  const int tile = 2 * warp + (lane >> 4), g = lane & 15;
  // store-phase identity: queries warp*32 + it*4 + qq, chunk c of 8
  const int qq = lane >> 3, chunk = lane & 7;
  const int pchunk = chunk ^ ((warp >> 1) & 7);  // physical 16-byte chunk of logical chunk `chunk`
  const bool swap_pairs = warp & 1;              // words k and k^2 swapped inside a chunk
  uint32_t cnt[8];
#pragma unroll
  for (int i = 0; i < 8; i++) cnt[i] = 0;

  // Positions are found one block ahead, inside the mask phase: even warps
  // before their masks, odd warps after, so the dependent shared-memory
  // loads of the boundary search overlap other warps' mask arithmetic.  The
  // table word offsets wait in registers as 16-bit pairs until the next
  // phase A writes them to the position buffer.  With up to 4 columns the
  // column values are loaded one more block ahead.
  constexpr bool kPrefetch = CMAX <= 4;
  uint32_t val[2][CMAX];             // column values of this thread's two rows
  uint32_t offn[2][(CMAX + 1) / 2];  // their table word offsets, two per register
  auto load_values = [&](uint64_t b) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const uint64_t row = b * kV4Rows + threadIdx.x + h * kV4Threads;
#pragma unroll
      for (int c = 0; c < CMAX; c++) val[h][c] = (c < C && row < p.nrows) ? __ldg(p.col[c] + row) : 0u;
    }
  };
  auto find_offsets = [&](uint64_t b) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const bool in = b * kV4Rows + threadIdx.x + h * kV4Threads < p.nrows;
      uint32_t off[CMAX];
#pragma unroll
      for (int c = 0; c < CMAX; c++)
        off[c] = c < C ? p.tab_off[c] + (in ? position(p, blob, c, val[h][c]) : 0u) * kV4Groups : 0u;
#pragma unroll
      for (int c = 0; c < CMAX; c += 2) offn[h][c / 2] = off[c] | (c + 1 < CMAX ? off[c + 1] << 16 : 0u);
    }
  };
  auto put_offsets = [&]() {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int r = threadIdx.x + h * kV4Threads;
      V4Pos<CMAX> *dst = posbuf + (r + (r >> 5)) * CMAX;
      if (CMAX <= 4) {
        *reinterpret_cast<uint4 *>(dst) = make_uint4(offn[h][0] & 0xFFFF, offn[h][0] >> 16,
                                                     offn[h][1 % ((CMAX + 1) / 2)] & 0xFFFF,
                                                     offn[h][1 % ((CMAX + 1) / 2)] >> 16);
      } else {
#pragma unroll
        for (int c = 0; c < CMAX; c += 4)
          *reinterpret_cast<uint2 *>(dst + c) = make_uint2(offn[h][c / 2], offn[h][c / 2 + 1]);
      }
    }
  };

  const uint64_t nblocks = p.nblocks, step = gridDim.x;
  uint64_t blk = p.block_begin + blockIdx.x;
  uint64_t prev = ~0ull;  // block whose stage is waiting to be stored
  if (blk < nblocks) {
    load_values(blk);
    find_offsets(blk);
    if (kPrefetch && blk + step < nblocks) load_values(blk + step);
  }
  while (true) {
    // ---- phase A: offsets of block `blk` to shared memory, store of block `prev` ----
    if (blk < nblocks) put_offsets();
    if (prev != ~0ull) {
      const uint64_t word0 = prev * kV4Tiles;
      const bool full = p.vec_store && word0 + kV4Tiles <= p.words;
#pragma unroll
      for (int it = 0; it < 8; it++) {
        const int q = warp * 32 + it * 4 + qq;
        const int32_t sq = slot_query[q];
        uint4 v = *reinterpret_cast<const uint4 *>(stage + q * kV4Tiles + pchunk * 4);
        if (swap_pairs) v = make_uint4(v.z, v.w, v.x, v.y);
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
    // ---- phase B: masks, transpose, stage of `blk`; offsets of the next block ----
    const uint64_t nxt = blk + step;
    auto ahead = [&]() {
      if (nxt < nblocks) {
        if (!kPrefetch) load_values(nxt);
        find_offsets(nxt);
        if (kPrefetch && nxt + step < nblocks) load_values(nxt + step);
      }
    };
    if (!(warp & 1)) ahead();
    {
      const uint64_t tile_row0 = blk * kV4Rows + (uint64_t)tile * 32;
      const uint32_t *tabg = blob + g;
      uint32_t acc[32];
#pragma unroll
      for (int r = 0; r < 32; r++) {
        const int row = tile * 32 + r;
        const V4Pos<CMAX> *pr = posbuf + (row + (row >> 5)) * CMAX;
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
            off[c + 1] = pv.x >> 16;
            off[c + 2] = pv.y & 0xFFFF;
            off[c + 3] = pv.y >> 16;
          }
        }
        uint32_t a = 0xFFFFFFFFu;
#pragma unroll
        for (int c = 0; c < CMAX; c++)
          if (c < C) a &= tabg[off[c]];
        acc[31 - r] = a;  // reversed: after the transpose row 0 is the MSB
      }
      transpose32(acc);
      if (tile_row0 + 32 > p.nrows) {
        const uint64_t valid = tile_row0 < p.nrows ? p.nrows - tile_row0 : 0;
        const uint32_t vm = valid >= 32 ? 0xFFFFFFFFu : (valid ? ~(0xFFFFFFFFu >> valid) : 0u);
#pragma unroll
        for (int j = 0; j < 32; j++) acc[j] &= vm;
      }
      const int col = tile ^ (2 * g);
#pragma unroll
      for (int j = 0; j < 32; j++) stage[(32 * g + j) * kV4Tiles + col] = acc[j];
    }
    if (warp & 1) ahead();
    __syncthreads();
    prev = blk;
    blk = nxt;
  }
  // counts: lanes with the same qq hold partial counts of the same queries
#pragma unroll
  for (int it = 0; it < 8; it++) {
    uint32_t c = cnt[it];
    c += __shfl_xor_sync(kFull, c, 1);
    c += __shfl_xor_sync(kFull, c, 2);
    c += __shfl_xor_sync(kFull, c, 4);
    const int q = warp * 32 + it * 4 + qq;
    const int32_t sq = slot_query[q];
    if (chunk == 0 && sq >= 0 && c) atomicAdd(p.counts + sq, (unsigned long long)c);
  }
}
