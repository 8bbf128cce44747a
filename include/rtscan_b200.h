/*
 * rtscan_b200.h -- C-ABI of the B200 multi-column range-predicate scan.
 *
 * This is the drop-in boundary for RTScan's scan path (AntaresAlice/RTScan).
 * The reference has no library ABI: its path sits behind driver main()s, the
 * column-file and scan_cmd formats, and a set of C-linkage-style CUDA host
 * functions (bindex.h:366-376, rt.h:337-345).  Each entry point below names
 * the reference interface it replaces.
 *
 * Conventions (all verified against the reference):
 *   - Columns are uint32 values; a column file holds `ncols` columns of
 *     `nrows` little-endian uint32 values back to back, no header
 *     (getDataFromFile, bindex_cuda.cpp:1269-1286).
 *   - A result bitmap is rts_bitmap_words(nrows) 32-bit words.  Row i is bit
 *     31-(i%32) of word i>>5 ("MSB-first", bindex.cpp:269,1217;
 *     cuda_and.cu:94-96).  Bits past row nrows-1 are always zero.
 *   - A query is a conjunction of terms lo <= column <= hi (inclusive).  The
 *     reference operators lt/le/gt/ge/eq/bt (raw_scan, bindex.cpp:1851-1892)
 *     are lowered to that form by rts_lower_op; a term with lo > hi matches
 *     nothing.
 *   - Every call returns an rts_status: 0 on success, a negative code on
 *     failure with a message from rts_last_error().  Nothing here calls
 *     exit() (the reference does, e.g. cuda_and.cu:528-546).
 *   - `stream` arguments are cudaStream_t values passed as void* (NULL = the
 *     legacy default stream).  *_async calls only enqueue work.
 *
 * Threading: one rts_ctx per host thread, except the rts_server_* calls,
 * which are safe from many producer threads.
 */
#ifndef RTSCAN_B200_H_
#define RTSCAN_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RTS_API __attribute__((visibility("default")))

/* ---- status codes ------------------------------------------------------ */
typedef int32_t rts_status;
#define RTS_OK 0
#define RTS_ERR_ARG (-1)      /* bad argument (null pointer, size, column index) */
#define RTS_ERR_CUDA (-2)     /* a CUDA call failed; message names it */
#define RTS_ERR_NOMEM (-3)    /* device or host allocation failed */
#define RTS_ERR_IO (-4)       /* file missing, short or unreadable */
#define RTS_ERR_PARSE (-5)    /* malformed scan_cmd text */
#define RTS_ERR_STATE (-6)    /* call not valid in this state (no columns, no index) */
#define RTS_ERR_TIMEOUT (-7)  /* a bounded wait ran out */
#define RTS_ERR_FULL (-8)     /* admission refused: queue or result memory full */
#define RTS_ERR_NODEV (-9)    /* no CUDA device, or not an sm_100 device */
#define RTS_ERR_CANCELLED (-10) /* the request was cancelled */

/* ---- operators: same order as the reference's OPERATOR enum (bindex.h:200-207) */
#define RTS_OP_EQ 0
#define RTS_OP_LT 1
#define RTS_OP_GT 2
#define RTS_OP_LE 3
#define RTS_OP_GE 4
#define RTS_OP_BT 5 /* t1 < x < t2, exclusive, bounds swapped when t1 > t2 */

/* One conjunct of a query: lo <= column <= hi (inclusive). */
typedef struct rts_term {
  int32_t column;
  uint32_t lo;
  uint32_t hi;
} rts_term;

typedef struct rts_ctx rts_ctx;
typedef struct rts_qset rts_qset;
typedef struct rts_server rts_server;

/* ---- errors and library info ------------------------------------------- */

/* Message of the last failed call on `ctx`, or of the calling thread's last
 * failed context-free call when ctx is NULL.  Never NULL. */
RTS_API const char *rts_last_error(const rts_ctx *ctx);
/* Library version string, e.g. "rtscan_b200 0.1 sm_100a". */
RTS_API const char *rts_version(void);
/* Words of a result bitmap for `nrows` rows: ceil(nrows/32)
 * (bits_num_needed, bindex.h:334-337). */
RTS_API uint64_t rts_bitmap_words(uint64_t nrows);

/* ---- operator lowering and scan_cmd parsing ----------------------------- */

/* Lower one reference operator to an inclusive range (replaces the operator
 * dispatch of raw_scan, bindex.cpp:1851-1892, without the reference's
 * overflow at the domain edges, bindex.cpp:1419-1427,1478-1487).
 * *nonempty is 0 when no value can match (lt 0, gt 4294967295, bt a b with
 * b <= a+1 after swapping). */
RTS_API rts_status rts_lower_op(int32_t op, uint32_t t1, uint32_t t2, uint32_t *lo, uint32_t *hi,
                                int32_t *nonempty);

/* Parse scan_cmd text (replaces the query loops of bindex.cpp:2165-2189,
 * bindex_cuda.cpp:1834-1854 and rtscan.cpp:992-1035 with stringSplit and
 * get_target_numbers, bindex.cpp:238-245,1840-1849).  `ncols` consecutive
 * lines form one conjunctive query, line c applying to column c; a line
 * `exit` (or the end of the text) ends the list and text after it is
 * ignored.  Each line is `<op> <t1>[,<t1>...] [<t2>[,<t2>...]]`, numbers
 * parsed as doubles and converted like the reference's (CODE)stod(..).  A
 * comma list of targets expands the query into one query per target
 * position.  Returns RTS_ERR_PARSE with the line number on malformed text. */
RTS_API rts_status rts_parse_scan_cmd(const char *text, uint64_t len, int32_t ncols, rts_qset **out);
RTS_API int32_t rts_qset_size(const rts_qset *qs);
/* Terms of query i (pointer valid until rts_qset_free).  *empty is 1 when
 * some term can never match (then the result is all zeros). */
RTS_API rts_status rts_qset_query(const rts_qset *qs, int32_t i, const rts_term **terms, int32_t *nterms,
                                  int32_t *empty);
/* The parsed operator of query i, column c, as written in the text. */
RTS_API rts_status rts_qset_line(const rts_qset *qs, int32_t i, int32_t c, int32_t *op, uint32_t *t1,
                                 uint32_t *t2);
RTS_API void rts_qset_free(rts_qset *qs);

/* ---- context and resident columns --------------------------------------- */

/* Open a context on CUDA device `device` (replaces the hard-coded
 * cudaSetDevice(0) of every cuda_and.cu entry point, e.g. cuda_and.cu:265). */
RTS_API rts_status rts_open(int32_t device, rts_ctx **out);
RTS_API void rts_close(rts_ctx *ctx);
/* Copy `ncols` host columns of `nrows` values into HBM, where they stay
 * resident (the rawDataInGPU upload of init_bindex_in_GPU,
 * bindex_cuda.cpp:192-194).  Replaces any earlier table and index. */
RTS_API rts_status rts_load_columns(rts_ctx *ctx, const uint32_t *const *host_cols, int32_t ncols,
                                    uint64_t nrows);
/* Read a column file (format above) into HBM (getDataFromFile,
 * bindex_cuda.cpp:1269-1286; get_data_from_file, rtscan.cpp:336-356).
 * nrows == 0 takes file size / (4*ncols). */
RTS_API rts_status rts_load_file(rts_ctx *ctx, const char *path, int32_t ncols, uint64_t nrows);
/* Borrow columns that already live on the context's device (no copy; the
 * caller keeps them alive until the next load or rts_close). */
RTS_API rts_status rts_attach_columns(rts_ctx *ctx, const uint32_t *const *dev_cols, int32_t ncols,
                                      uint64_t nrows);
RTS_API uint64_t rts_nrows(const rts_ctx *ctx);
RTS_API int32_t rts_ncols(const rts_ctx *ctx);
RTS_API int32_t rts_device(const rts_ctx *ctx);
RTS_API int32_t rts_sm_count(const rts_ctx *ctx);
RTS_API const uint32_t *rts_column_ptr(const rts_ctx *ctx, int32_t column);
/* Number of kernels this context has launched so far. */
RTS_API uint64_t rts_kernel_launches(const rts_ctx *ctx);

/* ---- single-query scans -------------------------------------------------- */

/* Fused conjunctive scan: one pass that reads every referenced column once,
 * compares lo <= x <= hi in registers, ANDs the terms and writes the packed
 * bitmap plus its popcount.  Replaces the per-column sieve copies, the
 * C-1 GPUbitAndWithCuda passes (merge_with_GPU, bindex_cuda.cpp:1662-1706;
 * cuda_and.cu:255-296) and the CPU hit count (compare_bitmap,
 * bindex.cpp:1959-1978).  dev_bitmap: rts_bitmap_words(nrows) words on the
 * device; *dev_count: one uint64 on the device, overwritten. */
RTS_API rts_status rts_scan_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap,
                                  uint64_t *dev_count, void *stream);
/* Same result by separate passes: one predicate pass per column into its own
 * bitmap, then C-1 AND passes, then a popcount pass -- the structure of the
 * reference's GPU path (bitmap_copy* + bit_andKernel, cuda_and.cu:13-61),
 * kept as the comparison the multi-column benchmark asks for.  Uses
 * context-owned scratch bitmaps. */
RTS_API rts_status rts_scan_separate_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms,
                                           uint32_t *dev_bitmap, uint64_t *dev_count, void *stream);
/* Blocking scan into host memory: the best device plan for the query, then
 * the bitmap copied to `host_bitmap` (rts_bitmap_words(nrows) words; pinned
 * memory is fastest) and the count to *count.  host_bitmap may be NULL to
 * fetch the count only.  (The result D2H of bindex_cuda.cpp:1932-1946.) */
RTS_API rts_status rts_scan(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *host_bitmap,
                            uint64_t *count);

/* ---- bitmap utilities ---------------------------------------------------- */
#define RTS_BM_AND 0    /* dst = a & b   (bit_andKernel, cuda_and.cu:13-20) */
#define RTS_BM_OR 1     /* dst = a | b   (bit_orKernel, cuda_and.cu:23-30) */
#define RTS_BM_COPY 2   /* dst = a       (bitmap_copyKernel, cuda_and.cu:34-41) */
#define RTS_BM_NOT 3    /* dst = ~a      (bitmap_copyNegationKernel, cuda_and.cu:45-52) */
#define RTS_BM_ANDNOT 4 /* dst = b & ~a  (bitmap_copySIMDKernel, cuda_and.cu:54-61) */
#define RTS_BM_FILL 5   /* dst = value   (bitmap_memsetKernel, cuda_and.cu:65-72) */
/* Element-wise bitmap op over `words` device words (replaces
 * GPUbit{And,Or,Copy,CopyNegation,CopySIMD,Memset}WithCuda, bindex.h:367-372).
 * dst may alias a.  `value` is used by RTS_BM_FILL only. */
RTS_API rts_status rts_bitmap_op_async(rts_ctx *ctx, int32_t op, uint32_t *dst, const uint32_t *a,
                                       const uint32_t *b, uint64_t words, uint32_t value, void *stream);
/* Popcount of the first `nbits` bits of a device bitmap into *dev_count. */
RTS_API rts_status rts_bitmap_count_async(rts_ctx *ctx, const uint32_t *bitmap, uint64_t nbits,
                                          uint64_t *dev_count, void *stream);

/* ---- BinDex: sieve + refine ---------------------------------------------- */

/* Build the BinDex index of one column on the GPU (replaces init_bindex,
 * bindex.cpp:599-671, and init_bindex_in_GPU, bindex_cuda.cpp:164-282):
 * sorted values and positions, K equal-count areas with the reference's
 * duplicate rule, and K-1 filter vectors fv[k] = (x < start value of area
 * k+1).  K in [2, 4096]; the reference's default is 128 (VAREA_N). */
RTS_API rts_status rts_build_bindex(rts_ctx *ctx, int32_t column, int32_t K);
RTS_API rts_status rts_drop_bindex(rts_ctx *ctx, int32_t column);
/* Area start values and their sorted positions (lower bounds) of a built
 * index, for inspection: starts[K], first_rank[K] on the host. */
RTS_API rts_status rts_bindex_areas(const rts_ctx *ctx, int32_t column, uint32_t *starts,
                                    uint64_t *first_rank, int32_t K);
/* Copy filter vector k (0 <= k < K-1) of a built index, rts_bitmap_words(nrows)
 * words, into host memory (the filterVectors[k] of bindex.h:311). */
RTS_API rts_status rts_bindex_filter_vector(rts_ctx *ctx, int32_t column, int32_t k, uint32_t *host_out);
/* Conjunctive query through the indexes: a sieve that ANDs 1-2 filter
 * vectors per term, then one refine launch that re-tests every row whose
 * sieve bit may be wrong (rows between a bound and its filter-vector
 * boundary, read from the sorted positions) on all terms, and fixes the bit
 * and the count.  Replaces bindex_scan_{lt,gt,bt}_in_GPU (bindex_cuda.cpp:
 * 903-1115), special_eq_scan (1450-1504), refine_with_Cuda (1506-1660) and
 * GPURefine{,Eq}AreaWithCuda (cuda_and.cu:510-812).  Every term's column
 * must have an index. */
RTS_API rts_status rts_bindex_scan_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms,
                                         uint32_t *dev_bitmap, uint64_t *dev_count, void *stream);

/* Save a column's BinDex to a file and load it back into a context whose
 * resident column is the same (no reference counterpart: the reference
 * rebuilds every index at start-up, bindex_cuda.cpp:1769-1781).  The file
 * carries a versioned header, checksums of every array (verified on load)
 * and the index's K and row count; loading also checks the sorted order
 * against the resident column and fails with RTS_ERR_PARSE on any mismatch.
 * rts_bindex_file_info reads only the header (no GPU needed). */
RTS_API rts_status rts_save_bindex(rts_ctx *ctx, int32_t column, const char *path);
RTS_API rts_status rts_load_bindex(rts_ctx *ctx, int32_t column, const char *path);
RTS_API rts_status rts_bindex_file_info(const char *path, int32_t *K, uint64_t *nrows);

/* ---- batched scans -------------------------------------------------------- */

/* Many queries in one pass (no reference counterpart; the reference runs one
 * query per loop iteration, bindex_cuda.cpp:1827-1986).  Queries are CSR:
 * query q owns terms[offsets[q] .. offsets[q+1]).  Query q's bitmap is
 * dev_bitmaps + q*stride_words (stride_words >= rts_bitmap_words(nrows));
 * its count is dev_counts[q].  The persistent kernel streams each column
 * chunk from HBM once and evaluates every query on it. */
RTS_API rts_status rts_scan_batch_async(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets,
                                        int32_t nqueries, uint32_t *dev_bitmaps, uint64_t stride_words,
                                        uint64_t *dev_counts, void *stream);
/* Batched scan over host-resident columns into host bitmaps: uploads the
 * `ncols` columns of `nrows` values (pinned host memory is fastest), runs
 * the batched passes, and writes every query's bitmap (host_bitmaps +
 * q*stride_words) and count (host_counts[q]), the download of each row
 * chunk overlapping the next chunk's pass (sparse chunks of a bitmap are
 * sent as a nonzero-word mask and the nonzero words, expanded by host
 * threads).  Blocking.  The
 * context's resident table is left as it was.  (The reference's per-query
 * upload-scan-download loop, bindex_cuda.cpp:1771-1946.) */
RTS_API rts_status rts_scan_batch_host(rts_ctx *ctx, const uint32_t *const *host_cols, int32_t ncols,
                                       uint64_t nrows, const rts_term *terms, const int32_t *offsets,
                                       int32_t nqueries, uint32_t *host_bitmaps, uint64_t stride_words,
                                       uint64_t *host_counts);
/* Bytes the context's last rts_scan_batch_host call moved host to device
 * (columns, plan) and device to host (bitmaps: a query's row chunk whose
 * nonzero-word mask, one bit per word, and nonzero words take at most 3/8
 * of its words travels as those, and the call expands it into
 * host_bitmaps; counts).  Zero before the first call. */
RTS_API rts_status rts_host_transfer_bytes(const rts_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes);
/* The same queries with one fused-scan launch per query (the baseline the
 * batched kernel is measured against). */
RTS_API rts_status rts_scan_each_async(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets,
                                       int32_t nqueries, uint32_t *dev_bitmaps, uint64_t stride_words,
                                       uint64_t *dev_counts, void *stream);

/* ---- prepared batches (CUDA graphs) -------------------------------------- */
typedef struct rts_prepared rts_prepared;
/* Plan a batch once and capture all of its launches (count reset, fills,
 * fused launches, one batched kernel per pass) into a CUDA graph writing
 * dev_bitmaps / dev_counts as rts_scan_batch_async would.  Re-prepare after
 * reloading the table. */
RTS_API rts_status rts_batch_prepare(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets,
                                     int32_t nqueries, uint32_t *dev_bitmaps, uint64_t stride_words,
                                     uint64_t *dev_counts, rts_prepared **out);
/* Replay a prepared batch on `stream` (one graph launch). */
RTS_API rts_status rts_batch_launch(rts_prepared *p, void *stream);
RTS_API void rts_batch_release(rts_prepared *p);

/* ---- batched-kernel launch shape and its autotuner ------------------------ */
typedef struct rts_batch_config {
  int32_t variant;              /* 4 (default): passes of up to 512 queries over CTA-wide row
                                   blocks, each pass in the smallest of the 128-, 256- and
                                   512-slot shapes that holds it, passes of at most 20 queries
                                   tested term by term, and passes of one query (or two or
                                   three with at most six terms) run as one fused scan per
                                   query; 3: 256-query passes, one 256-row block per warp */
  int32_t warps_per_cta;        /* 8 or 16.  Variant 4: CTA-wide blocks of 32 x 16 x warps / (slot
                                   groups) rows, two 8-warp CTAs per SM when the pass's tables
                                   leave room; variant 3: each warp stages 8 KiB of result words */
  int32_t max_queries_per_pass; /* 1..512 (variant 4), 1..256 (variant 3) */
  uint32_t table_budget_bytes;  /* shared memory a pass may use for its mask tables: 4 KiB up to
                                   136 KiB (variant 4), 88 KiB (variant 3, 16 warps), 140 KiB (8 warps) */
} rts_batch_config;
RTS_API rts_status rts_set_batch_config(rts_ctx *ctx, const rts_batch_config *cfg);
RTS_API rts_status rts_get_batch_config(const rts_ctx *ctx, rts_batch_config *cfg);
/* Time every candidate launch shape on the table's first rows (enough that
 * the batch's bitmaps take at most a quarter of the free device memory,
 * between 2^24 and 2^27 rows) with these queries, keep the fastest for this context, and
 * report it in *best (may be NULL).  With a cache_path, a previous result for
 * the same GPU, SM count, column count, table size and batch size is reused
 * and new results are appended. */
RTS_API rts_status rts_autotune_batch(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets,
                                      int32_t nqueries, const char *cache_path, rts_batch_config *best);
/* The last rts_autotune_batch of this context as JSON text: the sample rows,
 * every candidate shape with its time per call on the sample, the best and
 * the default shape's times ({"cached": true} when the cache answered; empty
 * before any tuning).  Copies at most size-1 bytes and a terminating NUL into
 * buf (may be NULL) and sets *needed (may be NULL) to the full length + 1.
 * No reference counterpart (its launch shape is fixed at compile time,
 * Makefile:31-58). */
RTS_API rts_status rts_autotune_report(const rts_ctx *ctx, char *buf, uint64_t size, uint64_t *needed);

/* ---- serving: continuous batching over resident columns ----------------- */
/* No reference counterpart (the reference drivers answer one query at a time,
 * bindex_cuda.cpp:1827-1986).  A server owns a worker thread that runs the
 * batched kernel as a circular scan over segments of the context's table:
 * requests are admitted into result slots as slots free up, join the scan
 * at the next segment, and are done when the scan has covered every
 * segment once for them.  While a server runs, its context must not be used
 * for other calls. */
typedef struct rts_server_config {
  int32_t max_active;         /* result slots (bitmap + count each); default 512 */
  int32_t max_queue;          /* requests waiting for a slot before RTS_ERR_FULL; default 65536 */
  uint64_t segment_rows;      /* rows per scan step, a multiple of 4096; default 2^22 */
  int32_t max_inflight_steps; /* steps queued on the GPU at once; default 3 */
} rts_server_config;

typedef struct rts_server_stats {
  uint64_t submitted, completed, rejected, cancelled, steps, queued;
  uint32_t active;
  double p50_ms, p99_ms, p999_ms, max_ms, mean_ms; /* submit-to-done latency of completed requests */
  uint64_t plans;       /* batch plans made for the active set */
  double plan_ms_total; /* host time spent making and uploading them */
} rts_server_stats;

/* cfg may be NULL (defaults); zero fields take their defaults.  Beside the
 * max_active result bitmaps the server holds 32 bytes per segment row for
 * the shared positions of its passes (268 MB for 2^23-row segments), or
 * runs without them when that memory is not there. */
RTS_API rts_status rts_server_start(rts_ctx *ctx, const rts_server_config *cfg, rts_server **out);
/* Queue one conjunctive query; safe from many threads.  RTS_ERR_FULL when the
 * queue holds max_queue requests. */
RTS_API rts_status rts_server_submit(rts_server *srv, const rts_term *terms, int32_t nterms, uint64_t *ticket);
RTS_API rts_status rts_server_poll(rts_server *srv, uint64_t ticket, int32_t *done, uint64_t *count);
/* Block until the request is done (RTS_ERR_TIMEOUT after timeout_ms). */
RTS_API rts_status rts_server_wait(rts_server *srv, uint64_t ticket, int32_t timeout_ms, uint64_t *count);
/* Copy a done request's bitmap (rts_bitmap_words(nrows) words; NULL to skip)
 * and count to the host and release its slot. */
RTS_API rts_status rts_server_fetch(rts_server *srv, uint64_t ticket, uint32_t *host_bitmap, uint64_t *count);
RTS_API rts_status rts_server_cancel(rts_server *srv, uint64_t ticket);
RTS_API rts_status rts_server_get_stats(rts_server *srv, rts_server_stats *stats);
/* Stop the worker and free the server (pending requests are dropped). */
RTS_API rts_status rts_server_stop(rts_server *srv);
/* Open-loop load replay for benchmarks: query q (CSR terms) is submitted
 * arrival_s[q] seconds after the call starts and released as soon as it is
 * done; latency_ms[q] gets its submit-to-done time (-1 if the queue was
 * full).  Blocks until all are done. */
RTS_API rts_status rts_server_replay(rts_server *srv, const rts_term *terms, const int32_t *offsets,
                                     int32_t nqueries, const double *arrival_s, double *latency_ms);

/* ---- rank encoding (remap.cpp) ---------------------------------------------- */
/* Replace every resident column by codes: row r's value becomes
 * encode_min + rank(r) * step, rank(r) its position in the column's stable
 * sorted order (ties by row id) and step = max(1, (encode_max - encode_min) /
 * nrows); the range must hold a code per row.  Indexes are dropped; borrowed
 * columns are not modified (the codes live in the context).  The
 * reference's normalEncode (remap.cpp:110-209) spreads the rows of one value
 * with rand(); this encoding is deterministic and order-preserving. */
RTS_API rts_status rts_encode_table(rts_ctx *ctx, uint32_t encode_min, uint32_t encode_max);
/* Rewrite terms on the original values into terms on the codes (encodeQuery,
 * remap.cpp:242-270, exact for every bound): out[i] selects on the encoded
 * table exactly the rows terms[i] selects on the original one; a term that
 * no value satisfies becomes the empty term lo = 1, hi = 0. */
RTS_API rts_status rts_encode_terms(rts_ctx *ctx, const rts_term *terms, int32_t nterms, rts_term *out);

/* ---- after the scan: row ids and aggregates --------------------------------- */
/* No reference counterpart: the reference stops at the bitmap and its hit
 * count, and its query files name the step that follows in a query engine
 * (TPC-H Q6, a filtered sum of l_extendedprice * l_discount,
 * test/scan_cmd_1e8-1c.txt:48-54). */

/* Ascending row ids of the set bits of an MSB-first bitmap of nrows bits
 * (nrows < 2^32; bits past nrows are ignored): at most `capacity` ids are
 * written to dev_rows, and *dev_count gets the number of set bits, so a
 * caller whose buffer was too small can size it and call again. */
RTS_API rts_status rts_bitmap_rows_async(rts_ctx *ctx, const uint32_t *dev_bitmap, uint64_t nrows,
                                         uint32_t *dev_rows, uint64_t capacity, uint64_t *dev_count,
                                         void *stream);
/* Sum over the set rows of dev_bitmap (rts_nrows(ctx) bits) of resident
 * column col_a, or of col_a x col_b when col_b >= 0: an exact 128-bit value
 * in dev_sum[0] (low 64 bits) and dev_sum[1] (high 64 bits). */
RTS_API rts_status rts_bitmap_sum_async(rts_ctx *ctx, const uint32_t *dev_bitmap, int32_t col_a, int32_t col_b,
                                        uint64_t *dev_sum, void *stream);
/* A conjunctive query and its aggregate in one pass, with no bitmap: the
 * hit count in *dev_count (may be NULL) and, when col_a >= 0, the 128-bit
 * sum of col_a (col_b < 0) or of col_a x col_b over the hits in dev_sum[0..1].
 * At most 8 distinct columns between the terms and the aggregate. */
RTS_API rts_status rts_scan_aggregate_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, int32_t col_a,
                                            int32_t col_b, uint64_t *dev_count, uint64_t *dev_sum, void *stream);

/* ---- allocation-free scan ------------------------------------------------ */

/* Largest row count rts_scan_separate_noalloc_async accepts (2^27 rows; its
 * scratch bitmap is a fixed 16 MiB device array). */
#define RTS_NOALLOC_MAX_ROWS (1ull << 27)
/* No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory -- an engine that hands all of HBM to its own pool
 * allocator at start-up, or a latency-critical caller that cannot afford
 * cudaMalloc's device-wide synchronisation -- this computes the result of
 * rts_scan_separate_async without a context and without allocating: plain
 * device column pointers in (`ncols` columns of `nrows` values on the
 * current device), caller-owned dev_bitmap (rts_bitmap_words(nrows) words)
 * and *dev_count out (required here, unlike rts_scan_separate_async),
 * asynchronously on `stream`.  Its scratch bitmap is a file-scope
 * __device__ array of RTS_NOALLOC_MAX_ROWS/8 bytes; nrows above
 * RTS_NOALLOC_MAX_ROWS is rejected with RTS_ERR_ARG.
 * Set-up: the first call on a device, with that device current, has the
 * CUDA runtime place the array and the kernels this call launches on the
 * device (the runtime allocates that memory then; device code loads
 * lazily) and looks up the array's device address.  From then on the
 * device holds them until the process exits and no call allocates.  So
 * make one warm-up call per device before reserving a pool that takes the
 * rest of the device, and before capturing any stream; a set-up that fails
 * returns RTS_ERR_CUDA and is retried by the next call.
 * Every call shares the one array and the array keeps the last call's
 * contents: the scan overwrites the words it reads, but calls that overlap
 * on the GPU (different streams, or several host threads) race on it. */
RTS_API rts_status rts_scan_separate_noalloc_async(const uint32_t *const *dev_cols, int32_t ncols,
                                                   uint64_t nrows, const rts_term *terms, int32_t nterms,
                                                   uint32_t *dev_bitmap, uint64_t *dev_count, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* RTSCAN_B200_H_ */
