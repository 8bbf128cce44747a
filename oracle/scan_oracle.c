/*
 * scan_oracle.c -- THE ORACLE.  Test infrastructure only.
 *
 * A plain-C, single-threaded restatement of the reference's CPU scan path
 * (AntaresAlice/RTScan, bindex.cpp).  It exists to check the CUDA product
 * path; nothing in the product links or calls it.  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it, and
 * only as the checker or as the timed CPU baseline.
 *
 * Two witnesses are restated:
 *   1. the scalar filter `raw_scan` (bindex.cpp:1851-1892) plus the
 *      conjunctive AND merge `refine_result_bitmap` (bindex.cpp:1259-1281)
 *      and the hit count of `compare_bitmap` (bindex.cpp:1959-1978).  This is
 *      the authority for every parity test.
 *   2. the BinDex index and its sieve+refine query (init_bindex,
 *      bindex.cpp:599-671; bindex_scan_{lt,le,gt,ge,bt,eq},
 *      bindex.cpp:1365-1691), including the reference's area/block choices.
 *
 * Parity is pinned by oracle/ref_harness.cpp, which links the reference's
 * own bindex.cpp (compiled unmodified from its source tree) and writes the
 * golden fixtures under tests/golden/.
 *
 * Bitmap convention (bindex.cpp:269,1217): row i is bit 31-(i%32) of 32-bit
 * word i>>5 ("MSB-first").
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EQ 0
#define ORC_LT 1
#define ORC_GT 2
#define ORC_LE 3
#define ORC_GE 4
#define ORC_BT 5

static inline uint32_t orc_bit(uint64_t i) { return 1u << (31 - (uint32_t)(i & 31)); }

/* refine() of bindex.cpp:1217 -- XOR one MSB-first bit. */
static inline void orc_flip(uint32_t *bm, uint64_t i) { bm[i >> 5] ^= orc_bit(i); }

uint64_t orc_words(uint64_t nbits) { return (nbits + 31) >> 5; }

/* raw_scan, bindex.cpp:1851-1892: per-row predicate; a hit XOR-sets the bit
 * (the reference calls refine(), so the bitmap must start at zero). */
void orc_raw_scan(const uint32_t *col, uint64_t n, int op, uint32_t t1, uint32_t t2, uint32_t *bitmap) {
  for (uint64_t i = 0; i < n; i++) {
    uint32_t x = col[i];
    int hit = 0;
    switch (op) {
      case ORC_LT: hit = x < t1; break;
      case ORC_LE: hit = x <= t1; break;
      case ORC_GT: hit = x > t1; break;
      case ORC_GE: hit = x >= t1; break;
      case ORC_EQ: hit = x == t1; break;
      case ORC_BT: hit = x > t1 && x < t2; break;
      default: break;
    }
    if (hit) orc_flip(bitmap, i);
  }
}

/* refine_result_bitmap, bindex.cpp:1259-1281: a[i] &= b[i] over words. */
void orc_and_bitmap(uint32_t *a, const uint32_t *b, uint64_t words) {
  for (uint64_t i = 0; i < words; i++) a[i] &= b[i];
}

/* Hit count of compare_bitmap, bindex.cpp:1959-1978: set bits among the
 * first nbits rows (tail bits past nbits are ignored, as the reference's
 * loop runs to len only). */
uint64_t orc_popcount(const uint32_t *bm, uint64_t nbits) {
  uint64_t full = nbits >> 5, c = 0;
  for (uint64_t w = 0; w < full; w++) c += (uint64_t)__builtin_popcount(bm[w]);
  uint32_t rem = (uint32_t)(nbits & 31);
  if (rem) c += (uint64_t)__builtin_popcount(bm[full] & ~(0xFFFFFFFFu >> rem));
  return c;
}

/* Operator lowering to the canonical inclusive range [lo,hi] (semantics of
 * raw_scan, bindex.cpp:1851-1892; bt swaps its bounds when t1>t2 as
 * raw_scan_entry does, bindex.cpp:1903-1905).  Returns 1 when the range is
 * non-empty, 0 when no value can match. */
int orc_lower_op(int op, uint32_t t1, uint32_t t2, uint32_t *lo, uint32_t *hi) {
  switch (op) {
    case ORC_LT: if (t1 == 0) return 0; *lo = 0; *hi = t1 - 1; return 1;
    case ORC_LE: *lo = 0; *hi = t1; return 1;
    case ORC_GT: if (t1 == 0xFFFFFFFFu) return 0; *lo = t1 + 1; *hi = 0xFFFFFFFFu; return 1;
    case ORC_GE: *lo = t1; *hi = 0xFFFFFFFFu; return 1;
    case ORC_EQ: *lo = t1; *hi = t1; return 1;
    case ORC_BT: {
      if (t1 > t2) { uint32_t t = t1; t1 = t2; t2 = t; }
      if ((uint64_t)t2 <= (uint64_t)t1 + 1) return 0;
      *lo = t1 + 1; *hi = t2 - 1; return 1;
    }
    default: return -1;
  }
}

/* Conjunctive scalar filter over inclusive ranges: the result raw_scan plus
 * the AND merge produce after lowering.  `bitmap` receives orc_words(n)
 * words, tail bits zero.  Returns the hit count. */
uint64_t orc_range_scan(const uint32_t *const *cols, int nterms, const uint32_t *lo, const uint32_t *hi,
                        uint64_t n, uint32_t *bitmap) {
  uint64_t words = orc_words(n), count = 0;
  memset(bitmap, 0, words * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; i++) {
    int hit = 1;
    for (int t = 0; t < nterms && hit; t++) {
      uint32_t x = cols[t][i];
      hit = (x >= lo[t]) && (x <= hi[t]);
    }
    if (hit) { bitmap[i >> 5] |= orc_bit(i); count++; }
  }
  return count;
}

/* ------------------------------------------------------------------------ */
/* BinDex restatement.                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint32_t n;            /* rows (bindex->length) */
  int K;                 /* number of virtual areas (VAREA_N, bindex.h:292) */
  int block_init;        /* blockInitSize = 3276 (bindex.cpp:199) */
  uint32_t *sval;        /* values in sorted order (data_sorted) */
  uint32_t *spos;        /* argsort positions (pos) */
  uint32_t *area_start;  /* areaStartIdx[K] (sorted index of each area's first row) */
  uint32_t *area_len;    /* rows in each area */
  uint32_t **fv;         /* K-1 filter vectors: fv[k] = (x < start value of area k+1) */
} orc_bindex;

static const uint32_t *g_sort_keys;
static int orc_cmp_pos(const void *a, const void *b) {
  uint32_t pa = *(const uint32_t *)a, pb = *(const uint32_t *)b;
  uint32_t va = g_sort_keys[pa], vb = g_sort_keys[pb];
  if (va != vb) return va < vb ? -1 : 1;
  return pa < pb ? -1 : (pa > pb);
}

/* gen_less_bits / set_fv_val_less, bindex.cpp:264-273,553-560. */
static void orc_set_fv_val_less(uint32_t *bm, const uint32_t *val, uint32_t compare, uint32_t n) {
  memset(bm, 0, orc_words(n) * sizeof(uint32_t));
  for (uint32_t i = 0; i < n; i++)
    if (val[i] < compare) bm[i >> 5] |= orc_bit(i);
}

static inline uint32_t area_sv(const orc_bindex *b, int a) { return b->sval[b->area_start[a]]; }
static inline int area_nblocks(const orc_bindex *b, int a) {
  /* init_area, bindex.cpp:410-427: blocks of block_init rows while more than
   * block_init rows remain, then one last block with the rest. */
  uint32_t len = b->area_len[a];
  int nb = 0;
  uint32_t i = 0;
  while (i + (uint32_t)b->block_init < len) { nb++; i += b->block_init; }
  return nb + 1;
}
static inline uint32_t blk_begin(const orc_bindex *b, int a, int blk) {
  return b->area_start[a] + (uint32_t)blk * (uint32_t)b->block_init;
}
static inline uint32_t blk_len(const orc_bindex *b, int a, int blk) {
  int nb = area_nblocks(b, a);
  if (blk < nb - 1) return (uint32_t)b->block_init;
  return b->area_len[a] - (uint32_t)(nb - 1) * (uint32_t)b->block_init;
}

/* init_bindex, bindex.cpp:599-671. Returns NULL on bad arguments. */
orc_bindex *orc_bindex_build(const uint32_t *data, uint32_t n, int K, int block_init) {
  if (n == 0 || K < 2 || block_init < 1 || (uint32_t)K > n) return NULL;
  orc_bindex *b = (orc_bindex *)calloc(1, sizeof(orc_bindex));
  b->n = n; b->K = K; b->block_init = block_init;
  b->sval = (uint32_t *)malloc((size_t)n * 4);
  b->spos = (uint32_t *)malloc((size_t)n * 4);
  for (uint32_t i = 0; i < n; i++) b->spos[i] = i;
  g_sort_keys = data;
  qsort(b->spos, n, sizeof(uint32_t), orc_cmp_pos);
  for (uint32_t i = 0; i < n; i++) b->sval[i] = data[b->spos[i]];

  b->area_start = (uint32_t *)malloc((size_t)K * 4);
  b->area_len = (uint32_t *)malloc((size_t)K * 4);
  uint32_t avg = n / (uint32_t)K;
  uint32_t *startv = (uint32_t *)malloc((size_t)K * 4);
  startv[0] = b->sval[0];
  b->area_start[0] = 0;
  for (int i = 1; i < K; i++) {
    /* duplicate rule, bindex.cpp:613-631 */
    uint32_t j = (uint32_t)i * avg;
    startv[i] = b->sval[j];
    if (startv[i] == startv[i - 1]) {
      b->area_start[i] = j;
    } else {
      while (b->sval[j] == startv[i]) j--;
      b->area_start[i] = j + 1;
    }
  }
  for (int i = 0; i < K; i++)
    b->area_len[i] = (i < K - 1 ? b->area_start[i + 1] : n) - b->area_start[i];
  b->fv = (uint32_t **)calloc((size_t)(K - 1), sizeof(uint32_t *));
  for (int k = 0; k < K - 1; k++) {
    b->fv[k] = (uint32_t *)malloc(orc_words(n) * 4);
    orc_set_fv_val_less(b->fv[k], data, area_sv(b, k + 1), n);
  }
  free(startv);
  return b;
}

void orc_bindex_free(orc_bindex *b) {
  if (!b) return;
  for (int k = 0; k < b->K - 1; k++) free(b->fv[k]);
  free(b->fv); free(b->sval); free(b->spos); free(b->area_start); free(b->area_len);
  free(b);
}

uint32_t orc_bindex_area_start_value(const orc_bindex *b, int a) { return area_sv(b, a); }
uint32_t orc_bindex_area_start_index(const orc_bindex *b, int a) { return b->area_start[a]; }

/* in_which_area, bindex.cpp:1138-1151. */
static int in_which_area(const orc_bindex *b, uint32_t compare) {
  if (compare < area_sv(b, 0)) return -1;
  for (int i = 0; i < b->K; i++) {
    uint32_t sv = area_sv(b, i);
    if (sv == compare) return i;
    if (sv > compare) return i - 1;
  }
  return b->K - 1;
}

/* in_which_block, bindex.cpp:1153-1177 (the linear search that returns). */
static int in_which_block(const orc_bindex *b, int a, uint32_t compare) {
  int nb = area_nblocks(b, a);
  int res = nb - 1;
  for (int i = 0; i < nb; i++) {
    uint32_t sv = b->sval[blk_begin(b, a, i)];
    if (sv == compare) { res = i; break; }
    if (sv > compare) { res = i - 1; break; }
  }
  if (res) {
    uint32_t last = b->sval[blk_begin(b, a, res - 1) + blk_len(b, a, res - 1) - 1];
    if (last == compare) res--;
  }
  return res;
}

/* on_which_pos, bindex.cpp:1201-1215: first index in the block whose value
 * is >= compare (block length if none). */
static uint32_t on_which_pos(const orc_bindex *b, int a, int blk, uint32_t compare) {
  uint32_t base = blk_begin(b, a, blk), lo = 0, hi = blk_len(b, a, blk);
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (b->sval[base + mid] >= compare) hi = mid; else lo = mid + 1;
  }
  return lo;
}

static void fill(uint32_t *r, uint64_t words, uint32_t v) {
  for (uint64_t i = 0; i < words; i++) r[i] = v;
}

/* copy_filter_vector (bindex.cpp:925-962) and copy_filter_vector_not
 * (bindex.cpp:964-1000). Out-of-range k fills all words, tail included. */
static void copy_fv(const orc_bindex *b, uint32_t *r, int k, int negate) {
  uint64_t w = orc_words(b->n);
  if (k < 0) { fill(r, w, negate ? 0xFFFFFFFFu : 0u); return; }
  if (k >= b->K - 1) { fill(r, w, negate ? 0u : 0xFFFFFFFFu); return; }
  for (uint64_t i = 0; i < w; i++) r[i] = negate ? ~b->fv[k][i] : b->fv[k][i];
}

/* copy_filter_vector_bt, bindex.cpp:1002-1048. */
static void copy_fv_bt(const orc_bindex *b, uint32_t *r, int kl, int kr) {
  uint64_t w = orc_words(b->n);
  if (kr < 0) { fill(r, w, 0); return; }
  if (kr >= b->K - 1) { copy_fv(b, r, kl, 1); return; }
  if (kl < 0) { copy_fv(b, r, kr, 0); return; }
  if (kl >= b->K - 1) { fill(r, w, 0); return; }
  for (uint64_t i = 0; i < w; i++) r[i] = ~b->fv[kl][i] & b->fv[kr][i];
}

/* copy_filter_vector_xor, bindex.cpp:1075-1136 (asserting branches return -1). */
static int copy_fv_xor(const orc_bindex *b, uint32_t *r, int kl, int kr) {
  uint64_t w = orc_words(b->n);
  if (kr < 0 || kr >= b->K - 1) return -1;
  if (kl < 0) { copy_fv(b, r, kr, 0); return 0; }
  if (kl >= b->K - 1) return -1;
  for (uint64_t i = 0; i < w; i++) r[i] = b->fv[kl][i] ^ b->fv[kr][i];
  return 0;
}

/* XOR-refine all rows of blocks [s,e) of area a (refine_positions_mt,
 * bindex.cpp:1225-1256), then the partial block (refine_positions). */
static void refine_blocks(const orc_bindex *b, uint32_t *r, int a, int s, int e) {
  for (int blk = s; blk < e; blk++) {
    uint32_t base = blk_begin(b, a, blk), len = blk_len(b, a, blk);
    for (uint32_t i = 0; i < len; i++) orc_flip(r, b->spos[base + i]);
  }
}
static void refine_range(const orc_bindex *b, uint32_t *r, int a, int blk, uint32_t from, uint32_t to) {
  uint32_t base = blk_begin(b, a, blk);
  for (uint32_t i = from; i < to; i++) orc_flip(r, b->spos[base + i]);
}

typedef struct { int area, blk, upper, s, e; uint32_t pos; } orc_locate;

static void locate(const orc_bindex *b, uint32_t compare, orc_locate *L) {
  L->area = in_which_area(b, compare);
  if (L->area < 0) return;
  L->blk = in_which_block(b, L->area, compare);
  L->pos = on_which_pos(b, L->area, L->blk, compare);
  int nb = area_nblocks(b, L->area);
  if (L->blk < nb / 2) { L->upper = 1; L->s = 0; L->e = L->blk; }
  else { L->upper = 0; L->s = L->blk + 1; L->e = nb; }
}

static void refine_located(const orc_bindex *b, uint32_t *r, const orc_locate *L) {
  refine_blocks(b, r, L->area, L->s, L->e);
  if (L->upper) refine_range(b, r, L->area, L->blk, 0, L->pos);
  else refine_range(b, r, L->area, L->blk, L->pos, blk_len(b, L->area, L->blk));
}

/* bindex_scan_lt, bindex.cpp:1365-1417. */
void orc_bindex_scan_lt(const orc_bindex *b, uint32_t *r, uint32_t compare) {
  orc_locate L;
  locate(b, compare, &L);
  if (L.area < 0) { fill(r, orc_words(b->n), 0); return; }
  copy_fv(b, r, L.upper ? L.area - 1 : L.area, 0);
  refine_located(b, r, &L);
}

/* bindex_scan_le, bindex.cpp:1419-1422 (compare+1 wraps at 2^32-1, as in
 * the reference). */
void orc_bindex_scan_le(const orc_bindex *b, uint32_t *r, uint32_t compare) {
  orc_bindex_scan_lt(b, r, compare + 1u);
}

/* bindex_scan_gt, bindex.cpp:1424-1476. */
void orc_bindex_scan_gt(const orc_bindex *b, uint32_t *r, uint32_t compare) {
  compare = compare + 1u;
  orc_locate L;
  locate(b, compare, &L);
  if (L.area < 0) { fill(r, orc_words(b->n), 0xFFFFFFFFu); return; }
  copy_fv(b, r, L.upper ? L.area - 1 : L.area, 1);
  refine_located(b, r, &L);
}

/* bindex_scan_ge, bindex.cpp:1478-1481. */
void orc_bindex_scan_ge(const orc_bindex *b, uint32_t *r, uint32_t compare) {
  orc_bindex_scan_gt(b, r, compare - 1u);
}

/* bindex_scan_bt, bindex.cpp:1483-1573 (exclusive both ends).  Returns -1
 * where the reference asserts. */
int orc_bindex_scan_bt(const orc_bindex *b, uint32_t *r, uint32_t c1, uint32_t c2) {
  if (!(c2 > c1)) return -1;
  c1 = c1 + 1u;
  orc_locate Ll, Lr;
  locate(b, c1, &Ll);
  if (Ll.area < 0) { fill(r, orc_words(b->n), 0xFFFFFFFFu); return 0; }
  locate(b, c2, &Lr);
  if (Lr.area < 0) return -1;
  copy_fv_bt(b, r, Ll.upper ? Ll.area - 1 : Ll.area, Lr.upper ? Lr.area - 1 : Lr.area);
  refine_located(b, r, &Ll);
  refine_located(b, r, &Lr);
  return 0;
}

/* bindex_scan_eq, bindex.cpp:1575-1691.  Returns -1 where the reference
 * asserts (a value below the column minimum, or an out-of-range filter
 * vector in the xor branch). */
int orc_bindex_scan_eq(const orc_bindex *b, uint32_t *r, uint32_t compare) {
  uint64_t w = orc_words(b->n);
  int area_idx = in_which_area(b, compare);
  if (area_idx < 0 || area_idx > b->K - 1) return -1;
  if (area_idx != b->K - 1 && area_sv(b, area_idx + 1) == compare) {
    orc_locate L0;
    locate(b, compare, &L0);
    uint32_t c1 = compare + 1u;
    int a1 = in_which_area(b, c1);
    if (a1 < 0) return -1;
    int blk1 = in_which_block(b, a1, c1);
    uint32_t pos1 = on_which_pos(b, a1, blk1, c1);
    int nb1 = area_nblocks(b, a1);
    orc_locate L1;
    L1.area = a1; L1.blk = blk1; L1.pos = pos1;
    if (a1 == 0 || (blk1 < nb1 / 2 && area_sv(b, a1 - 1) != area_sv(b, a1))) {
      L1.upper = 1; L1.s = 0; L1.e = blk1;
    } else {
      L1.upper = 0; L1.s = blk1 + 1; L1.e = nb1;
    }
    if (copy_fv_xor(b, r, L0.upper ? L0.area - 1 : L0.area, L1.upper ? L1.area - 1 : L1.area) != 0) return -1;
    refine_located(b, r, &L0);
    refine_located(b, r, &L1);
    return 0;
  }
  /* set_eq_bitmap_mt, bindex.cpp:1302-1328 */
  fill(r, w, 0);
  int blk0 = in_which_block(b, area_idx, compare);
  int nb = area_nblocks(b, area_idx);
  for (int blk = blk0; blk < nb; blk++) {
    uint32_t base = blk_begin(b, area_idx, blk), len = blk_len(b, area_idx, blk);
    if (b->sval[base] > compare) break;
    for (uint32_t j = 0; j < len && b->sval[base + j] <= compare; j++)
      if (b->sval[base + j] == compare) orc_flip(r, b->spos[base + j]);
  }
  return 0;
}

/* One reference op on one column: dispatch of exp_opt, bindex.cpp:2191-2227.
 * Returns -1 where the reference would assert. */
int orc_bindex_scan_op(const orc_bindex *b, uint32_t *r, int op, uint32_t t1, uint32_t t2) {
  switch (op) {
    case ORC_LT: orc_bindex_scan_lt(b, r, t1); return 0;
    case ORC_LE: orc_bindex_scan_le(b, r, t1); return 0;
    case ORC_GT: orc_bindex_scan_gt(b, r, t1); return 0;
    case ORC_GE: orc_bindex_scan_ge(b, r, t1); return 0;
    case ORC_EQ: return orc_bindex_scan_eq(b, r, t1);
    case ORC_BT:
      if (t1 > t2) { uint32_t t = t1; t1 = t2; t2 = t; }
      return orc_bindex_scan_bt(b, r, t1, t2);
    default: return -1;
  }
}

/* Filter vector k of a restated index (orc_words(n) words). */
const uint32_t *orc_bindex_fv(const orc_bindex *b, int k) {
  if (!b || k < 0 || k >= b->K - 1) return 0;
  return b->fv[k];
}
