// C-ABI implementation: context, resident columns, scan planning.
//
// Host side of the drop-in boundary declared in include/rtscan_b200.h.  The
// reference keeps this logic in its driver main()s and in process-global
// state guarded by a mutex (bindex_cuda.cpp:7-15, 1708-1995); here it is a
// context object, every failure is a status code, and nothing exits.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cstdint>
#include <new>
#include <string>
#include <vector>

#include "rts_internal.h"

using rts::Error;

namespace {
thread_local std::string g_err;

rts_status fail(rts_ctx *ctx, rts_status code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  g_err = msg;
  return code;
}

template <class F>
rts_status guarded(rts_ctx *ctx, F &&f) {
  try {
    return f();
  } catch (const Error &e) {
    return fail(ctx, e.code, e.what());
  } catch (const std::bad_alloc &) {
    return fail(ctx, RTS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(ctx, RTS_ERR_ARG, e.what());
  }
}

using rts::DeviceGuard;

void check_launch(rts_ctx *ctx, int n) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(RTS_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  ctx->launches += (uint64_t)n;
}

void need_ctx(rts_ctx *ctx) {
  if (!ctx) throw Error(RTS_ERR_ARG, "null context");
}

void need_table(rts_ctx *ctx) {
  need_ctx(ctx);
  if (ctx->cols.empty() || ctx->nrows == 0) throw Error(RTS_ERR_STATE, "no columns loaded");
}

void release_table(rts_ctx *ctx) {
  ctx->bindex.clear();
  ctx->encode.reset();
  if (ctx->owned) cudaFree(ctx->owned);
  ctx->owned = nullptr;
  ctx->owned_bytes = 0;
  ctx->cols.clear();
  ctx->nrows = 0;
  for (uint32_t *p : ctx->scratch_bm) cudaFree(p);
  ctx->scratch_bm.clear();
  ctx->scratch_words = 0;
}

// A query after validation: terms grouped per column with ranges
// intersected, always-true terms dropped.
struct Plan {
  bool empty = false;                 // some term can never match
  std::vector<rts::DevTerm> terms;    // remaining terms, one per column
  std::vector<int> columns;
};

Plan make_plan(rts_ctx *ctx, const rts_term *terms, int32_t nterms) {
  if (nterms < 0 || (nterms > 0 && !terms)) throw Error(RTS_ERR_ARG, "bad term list");
  Plan p;
  std::vector<int> order;
  std::vector<uint32_t> lo, hi;
  for (int i = 0; i < nterms; i++) {
    const rts_term &t = terms[i];
    if (t.column < 0 || t.column >= (int)ctx->cols.size())
      throw Error(RTS_ERR_ARG, "term " + std::to_string(i) + ": column " + std::to_string(t.column) +
                                   " out of range (table has " + std::to_string(ctx->cols.size()) + ")");
    if (t.lo > t.hi) p.empty = true;
    auto it = std::find(order.begin(), order.end(), (int)t.column);
    if (it == order.end()) {
      order.push_back(t.column);
      lo.push_back(t.lo);
      hi.push_back(t.hi);
    } else {
      size_t k = it - order.begin();
      lo[k] = std::max(lo[k], t.lo);
      hi[k] = std::min(hi[k], t.hi);
      if (lo[k] > hi[k]) p.empty = true;
    }
  }
  if (p.empty) return p;
  for (size_t k = 0; k < order.size(); k++) {
    if (lo[k] == 0 && hi[k] == 0xFFFFFFFFu) continue;  // always true
    p.terms.push_back({ctx->cols[order[k]], lo[k], hi[k] - lo[k]});
    p.columns.push_back(order[k]);
  }
  return p;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// Run the fused kernel over a plan, in passes of at most kFusedMaxTerms.
void fused(rts_ctx *ctx, const Plan &plan, uint32_t *out, unsigned long long *count, cudaStream_t s) {
  const uint64_t n = ctx->nrows;
  if (plan.empty || plan.terms.empty()) {
    rts::launch_fill_range(out, n, !plan.empty, count, ctx->sm_count, s);
    check_launch(ctx, 1);
    return;
  }
  if (count) RTS_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), s));
  const size_t T = plan.terms.size();
  int launches = 0;
  for (size_t first = 0; first < T; first += rts::kFusedMaxTerms) {
    rts::ScanParams p;
    memset(&p, 0, sizeof p);
    size_t cnt = std::min<size_t>(rts::kFusedMaxTerms, T - first);
    bool vec = true;
    for (size_t i = 0; i < cnt; i++) {
      p.t[i] = plan.terms[first + i];
      vec = vec && aligned16(p.t[i].col);
    }
    p.nterms = (int)cnt;
    p.and_into = first > 0;
    p.out = out;
    p.count = (first + cnt == T) ? count : nullptr;
    p.nrows = n;
    p.full_tiles = n / rts::kTileRows;
    rts::launch_scan_fused(p, vec, ctx->sm_count, s);
    launches++;
  }
  check_launch(ctx, launches);
}

uint32_t *scratch_bitmap(rts_ctx *ctx, size_t i) {
  const uint64_t words = rts::words_for(ctx->nrows);
  if (ctx->scratch_words != words) {
    for (uint32_t *p : ctx->scratch_bm) cudaFree(p);
    ctx->scratch_bm.clear();
    ctx->scratch_words = words;
  }
  while (ctx->scratch_bm.size() <= i) {
    uint32_t *p = nullptr;
    if (cudaMalloc(&p, std::max<uint64_t>(words, 4) * 4) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "scratch bitmap allocation failed");
    }
    ctx->scratch_bm.push_back(p);
  }
  return ctx->scratch_bm[i];
}

}  // namespace

rts_status rts::set_thread_error(rts_status code, const std::string &msg) {
  g_err = msg;
  return code;
}

unsigned long long *rts::small_device_buffer(rts_ctx *ctx) {
  if (!ctx->small_dev) {
    if (cudaMalloc(&ctx->small_dev, 256) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "device allocation failed");
    }
  }
  return reinterpret_cast<unsigned long long *>(ctx->small_dev);
}

rts_ctx::~rts_ctx() {
  release_table(this);
  if (plan_dev) cudaFree(plan_dev);
  if (plan_host) cudaFreeHost(plan_host);
  if (small_dev) cudaFree(small_dev);
  if (query_slots) cudaFree(query_slots);
  if (agg_dev) cudaFree(agg_dev);
  if (batch) rts::destroy_batch(batch);
  if (host_batch) rts::destroy_host_batch(host_batch);
}

extern "C" {

const char *rts_last_error(const rts_ctx *ctx) {
  if (ctx) return ctx->err.c_str();
  return g_err.c_str();
}

const char *rts_version(void) { return "rtscan_b200 0.1 sm_100a"; }

uint64_t rts_bitmap_words(uint64_t nrows) { return rts::words_for(nrows); }

rts_status rts_lower_op(int32_t op, uint32_t t1, uint32_t t2, uint32_t *lo, uint32_t *hi, int32_t *nonempty) {
  return guarded(nullptr, [&]() -> rts_status {
    if (!lo || !hi || !nonempty) return fail(nullptr, RTS_ERR_ARG, "null output pointer");
    *nonempty = 1;
    switch (op) {
      case RTS_OP_LT:
        if (t1 == 0) { *nonempty = 0; *lo = 1; *hi = 0; return RTS_OK; }
        *lo = 0; *hi = t1 - 1; return RTS_OK;
      case RTS_OP_LE: *lo = 0; *hi = t1; return RTS_OK;
      case RTS_OP_GT:
        if (t1 == 0xFFFFFFFFu) { *nonempty = 0; *lo = 1; *hi = 0; return RTS_OK; }
        *lo = t1 + 1; *hi = 0xFFFFFFFFu; return RTS_OK;
      case RTS_OP_GE: *lo = t1; *hi = 0xFFFFFFFFu; return RTS_OK;
      case RTS_OP_EQ: *lo = t1; *hi = t1; return RTS_OK;
      case RTS_OP_BT:
        if (t1 > t2) std::swap(t1, t2);
        if ((uint64_t)t2 <= (uint64_t)t1 + 1) { *nonempty = 0; *lo = 1; *hi = 0; return RTS_OK; }
        *lo = t1 + 1; *hi = t2 - 1; return RTS_OK;
      default: return fail(nullptr, RTS_ERR_ARG, "unknown operator " + std::to_string(op));
    }
  });
}

rts_status rts_open(int32_t device, rts_ctx **out) {
  return guarded(nullptr, [&]() -> rts_status {
    if (!out) throw Error(RTS_ERR_ARG, "null output pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Error(RTS_ERR_NODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) throw Error(RTS_ERR_ARG, "device index out of range");
    cudaDeviceProp prop;
    RTS_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0)
      throw Error(RTS_ERR_NODEV, std::string("device ") + prop.name + " is not sm_100 (this library is built for sm_100a)");
    auto *ctx = new rts_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    *out = ctx;
    return RTS_OK;
  });
}

void rts_close(rts_ctx *ctx) {
  if (!ctx) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  delete ctx;
  if (prev >= 0) cudaSetDevice(prev);
}

rts_status rts_load_columns(rts_ctx *ctx, const uint32_t *const *host_cols, int32_t ncols, uint64_t nrows) {
  rts::Range nvtx_range_("rts_load_columns");
  return guarded(ctx, [&]() -> rts_status {
    need_ctx(ctx);
    if (ncols < 1 || nrows == 0 || !host_cols) throw Error(RTS_ERR_ARG, "need ncols >= 1, nrows >= 1 and columns");
    for (int c = 0; c < ncols; c++)
      if (!host_cols[c]) throw Error(RTS_ERR_ARG, "null column pointer");
    DeviceGuard g(ctx->device);
    // Pad each column to whole 1024-row tiles plus 16-byte alignment; a
    // table that fits the previous allocation reuses it.
    const uint64_t stride = (nrows + rts::kTileRows - 1) / rts::kTileRows * rts::kTileRows;
    const size_t bytes = stride * ncols * sizeof(uint32_t);
    uint32_t *buf = nullptr;
    const size_t kept = ctx->owned_bytes;
    if (ctx->owned && kept >= bytes) {
      buf = ctx->owned;
      ctx->owned = nullptr;  // kept across release_table
    }
    release_table(ctx);
    if (buf) {
      ctx->owned_bytes = kept;
    } else {
      if (cudaMalloc(&buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw Error(RTS_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
      }
      ctx->owned_bytes = bytes;
    }
    ctx->owned = buf;
    ctx->col_stride = stride;
    for (int c = 0; c < ncols; c++) {
      uint32_t *dst = buf + stride * c;
      RTS_CUDA(cudaMemcpy(dst, host_cols[c], nrows * 4, cudaMemcpyHostToDevice));
      if (stride > nrows) RTS_CUDA(cudaMemset(dst + nrows, 0, (stride - nrows) * 4));
      ctx->cols.push_back(dst);
    }
    ctx->nrows = nrows;
    ctx->bindex.resize(ncols);
    return RTS_OK;
  });
}

rts_status rts_load_file(rts_ctx *ctx, const char *path, int32_t ncols, uint64_t nrows) {
  rts::Range nvtx_range_("rts_load_file");
  return guarded(ctx, [&]() -> rts_status {
    need_ctx(ctx);
    if (!path || ncols < 1) throw Error(RTS_ERR_ARG, "need a path and ncols >= 1");
    FILE *fp = fopen(path, "rb");
    if (!fp) throw Error(RTS_ERR_IO, std::string("cannot open ") + path);
    struct Closer { FILE *f; ~Closer() { fclose(f); } } closer{fp};
    if (fseeko(fp, 0, SEEK_END) != 0) throw Error(RTS_ERR_IO, "cannot seek");
    const uint64_t size = (uint64_t)ftello(fp);
    fseeko(fp, 0, SEEK_SET);
    if (nrows == 0) nrows = size / (4ull * ncols);
    if (nrows == 0 || size < 4ull * ncols * nrows)
      throw Error(RTS_ERR_IO, std::string(path) + ": file holds " + std::to_string(size) + " bytes, need " +
                                  std::to_string(4ull * ncols * nrows));
    DeviceGuard g(ctx->device);
    release_table(ctx);
    const uint64_t stride = (nrows + rts::kTileRows - 1) / rts::kTileRows * rts::kTileRows;
    uint32_t *buf = nullptr;
    if (cudaMalloc(&buf, stride * ncols * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(RTS_ERR_NOMEM, "device allocation failed");
    }
    ctx->owned = buf;
    ctx->owned_bytes = stride * ncols * sizeof(uint32_t);
    ctx->col_stride = stride;
    const size_t chunk = 1u << 24;  // values per staging copy
    uint32_t *stage = nullptr;
    RTS_CUDA(cudaMallocHost(&stage, chunk * 4));
    struct Freer { uint32_t *p; ~Freer() { cudaFreeHost(p); } } freer{stage};
    for (int c = 0; c < ncols; c++) {
      uint32_t *dst = buf + stride * c;
      for (uint64_t off = 0; off < nrows; off += chunk) {
        size_t m = (size_t)std::min<uint64_t>(chunk, nrows - off);
        if (fread(stage, 4, m, fp) != m) throw Error(RTS_ERR_IO, std::string(path) + ": short read");
        RTS_CUDA(cudaMemcpy(dst + off, stage, m * 4, cudaMemcpyHostToDevice));
      }
      if (stride > nrows) RTS_CUDA(cudaMemset(dst + nrows, 0, (stride - nrows) * 4));
      ctx->cols.push_back(dst);
    }
    ctx->nrows = nrows;
    ctx->bindex.resize(ncols);
    return RTS_OK;
  });
}

rts_status rts_attach_columns(rts_ctx *ctx, const uint32_t *const *dev_cols, int32_t ncols, uint64_t nrows) {
  return guarded(ctx, [&]() -> rts_status {
    need_ctx(ctx);
    if (ncols < 1 || nrows == 0 || !dev_cols) throw Error(RTS_ERR_ARG, "need ncols >= 1, nrows >= 1 and columns");
    DeviceGuard g(ctx->device);
    for (int c = 0; c < ncols; c++) {
      if (!dev_cols[c]) throw Error(RTS_ERR_ARG, "null column pointer");
      cudaPointerAttributes a;
      if (cudaPointerGetAttributes(&a, dev_cols[c]) != cudaSuccess || a.type != cudaMemoryTypeDevice ||
          a.device != ctx->device) {
        cudaGetLastError();
        throw Error(RTS_ERR_ARG, "column " + std::to_string(c) + " is not device memory of this context's device");
      }
    }
    release_table(ctx);
    for (int c = 0; c < ncols; c++) ctx->cols.push_back(dev_cols[c]);
    ctx->nrows = nrows;
    ctx->bindex.resize(ncols);
    return RTS_OK;
  });
}

uint64_t rts_nrows(const rts_ctx *ctx) { return ctx ? ctx->nrows : 0; }
int32_t rts_ncols(const rts_ctx *ctx) { return ctx ? (int32_t)ctx->cols.size() : 0; }
int32_t rts_device(const rts_ctx *ctx) { return ctx ? ctx->device : -1; }
int32_t rts_sm_count(const rts_ctx *ctx) { return ctx ? ctx->sm_count : 0; }
const uint32_t *rts_column_ptr(const rts_ctx *ctx, int32_t c) {
  if (!ctx || c < 0 || c >= (int)ctx->cols.size()) return nullptr;
  return ctx->cols[c];
}
uint64_t rts_kernel_launches(const rts_ctx *ctx) { return ctx ? ctx->launches.load() : 0; }

rts_status rts_scan_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap,
                          uint64_t *dev_count, void *stream) {
  rts::Range nvtx_range_("rts_scan_async");
  return guarded(ctx, [&]() -> rts_status {
    need_table(ctx);
    if (!dev_bitmap) throw Error(RTS_ERR_ARG, "null result bitmap");
    DeviceGuard g(ctx->device);
    Plan plan = make_plan(ctx, terms, nterms);
    fused(ctx, plan, dev_bitmap, reinterpret_cast<unsigned long long *>(dev_count), (cudaStream_t)stream);
    return RTS_OK;
  });
}

rts_status rts_scan_separate_async(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *dev_bitmap,
                                   uint64_t *dev_count, void *stream) {
  rts::Range nvtx_range_("rts_scan_separate_async");
  return guarded(ctx, [&]() -> rts_status {
    need_table(ctx);
    if (!dev_bitmap) throw Error(RTS_ERR_ARG, "null result bitmap");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    Plan plan = make_plan(ctx, terms, nterms);
    if (plan.empty || plan.terms.empty()) {
      fused(ctx, plan, dev_bitmap, reinterpret_cast<unsigned long long *>(dev_count), s);
      return RTS_OK;
    }
    const uint64_t n = ctx->nrows, words = rts::words_for(n);
    int launches = 0;
    for (size_t i = 0; i < plan.terms.size(); i++) {
      rts::ScanParams p;
      memset(&p, 0, sizeof p);
      p.t[0] = plan.terms[i];
      p.nterms = 1;
      p.out = i == 0 ? dev_bitmap : scratch_bitmap(ctx, 0);
      p.nrows = n;
      p.full_tiles = n / rts::kTileRows;
      rts::launch_scan_fused(p, aligned16(p.t[0].col), ctx->sm_count, s);
      launches++;
      if (i > 0) {
        rts::launch_bitmap_op(RTS_BM_AND, dev_bitmap, dev_bitmap, p.out, words, 0, ctx->sm_count, s);
        launches++;
      }
    }
    if (dev_count) {
      RTS_CUDA(cudaMemsetAsync(dev_count, 0, 8, s));
      rts::launch_bitmap_count(dev_bitmap, n, reinterpret_cast<unsigned long long *>(dev_count), ctx->sm_count, s);
      launches++;
    }
    check_launch(ctx, launches);
    return RTS_OK;
  });
}

rts_status rts_scan(rts_ctx *ctx, const rts_term *terms, int32_t nterms, uint32_t *host_bitmap, uint64_t *count) {
  rts::Range nvtx_range_("rts_scan");
  return guarded(ctx, [&]() -> rts_status {
    need_table(ctx);
    if (!count) throw Error(RTS_ERR_ARG, "null count pointer");
    DeviceGuard g(ctx->device);
    Plan plan = make_plan(ctx, terms, nterms);
    uint32_t *bm = scratch_bitmap(ctx, 1);
    unsigned long long *dcount = rts::small_device_buffer(ctx);
    cudaStream_t s = nullptr;
    bool indexed = !plan.empty && !plan.terms.empty();
    for (int c : plan.columns) indexed = indexed && c < (int)ctx->bindex.size() && ctx->bindex[c];
    if (indexed) {
      rts::bindex_query(ctx, terms, nterms, bm, dcount, s);
    } else {
      fused(ctx, plan, bm, dcount, s);
    }
    if (host_bitmap) RTS_CUDA(cudaMemcpyAsync(host_bitmap, bm, rts::words_for(ctx->nrows) * 4, cudaMemcpyDeviceToHost, s));
    unsigned long long c = 0;
    RTS_CUDA(cudaMemcpyAsync(&c, dcount, 8, cudaMemcpyDeviceToHost, s));
    RTS_CUDA(cudaStreamSynchronize(s));
    *count = c;
    return RTS_OK;
  });
}

rts_status rts_bitmap_op_async(rts_ctx *ctx, int32_t op, uint32_t *dst, const uint32_t *a, const uint32_t *b,
                               uint64_t words, uint32_t value, void *stream) {
  return guarded(ctx, [&]() -> rts_status {
    need_ctx(ctx);
    if (op < RTS_BM_AND || op > RTS_BM_FILL) throw Error(RTS_ERR_ARG, "unknown bitmap op");
    if (!dst || (op != RTS_BM_FILL && !a) || ((op == RTS_BM_AND || op == RTS_BM_OR || op == RTS_BM_ANDNOT) && !b))
      throw Error(RTS_ERR_ARG, "null bitmap");
    if (words == 0) return RTS_OK;
    DeviceGuard g(ctx->device);
    rts::launch_bitmap_op(op, dst, a, b, words, value, ctx->sm_count, (cudaStream_t)stream);
    check_launch(ctx, 1);
    return RTS_OK;
  });
}

rts_status rts_bitmap_count_async(rts_ctx *ctx, const uint32_t *bitmap, uint64_t nbits, uint64_t *dev_count,
                                  void *stream) {
  return guarded(ctx, [&]() -> rts_status {
    need_ctx(ctx);
    if (!bitmap || !dev_count) throw Error(RTS_ERR_ARG, "null pointer");
    DeviceGuard g(ctx->device);
    cudaStream_t s = (cudaStream_t)stream;
    RTS_CUDA(cudaMemsetAsync(dev_count, 0, 8, s));
    if (nbits) {
      rts::launch_bitmap_count(bitmap, nbits, reinterpret_cast<unsigned long long *>(dev_count), ctx->sm_count, s);
      check_launch(ctx, 1);
    }
    return RTS_OK;
  });
}

rts_status rts_scan_each_async(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int32_t nq,
                               uint32_t *dev_bitmaps, uint64_t stride_words, uint64_t *dev_counts, void *stream) {
  rts::Range nvtx_range_("rts_scan_each_async");
  return guarded(ctx, [&]() -> rts_status {
    need_table(ctx);
    if (nq < 0 || (nq > 0 && (!offsets || !dev_bitmaps))) throw Error(RTS_ERR_ARG, "bad batch arguments");
    if (stride_words < rts::words_for(ctx->nrows)) throw Error(RTS_ERR_ARG, "stride_words smaller than a bitmap");
    DeviceGuard g(ctx->device);
    for (int q = 0; q < nq; q++) {
      if (offsets[q + 1] < offsets[q] || offsets[q] < 0) throw Error(RTS_ERR_ARG, "offsets not ascending");
      Plan plan = make_plan(ctx, terms + offsets[q], offsets[q + 1] - offsets[q]);
      fused(ctx, plan, dev_bitmaps + (uint64_t)q * stride_words,
            dev_counts ? reinterpret_cast<unsigned long long *>(dev_counts + q) : nullptr, (cudaStream_t)stream);
    }
    return RTS_OK;
  });
}

}  // extern "C"
