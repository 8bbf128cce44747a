// Rank encoding of the resident table and the exact rewrite of query terms.
//
// The reference's RT driver can encode every column before indexing it
// (normalEncode, remap.cpp:110-209, used when ENCODE=1, rtscan.cpp:1069-1072):
// values are sorted, each row's value is replaced by its row's position in
// the sorted order scaled into [encode_min, encode_max), and query bounds are
// rewritten through the value -> first-code map (encodeQuery,
// remap.cpp:242-270).  Duplicate-heavy columns become dense and uniform,
// which is what BVH and BinDex area balance want.  The reference spreads the
// rows of one value with rand() (remap.cpp:35,234), so its encoding differs
// from run to run, and its rewrite of `gt` skips the first row above the
// bound.  Here:
//
//   * the sort is a stable device radix sort of (value, row id), so rows of
//     one value keep their row order and code(row) = encode_min +
//     rank(row) * step with step = max(1, (encode_max - encode_min) / n) is
//     deterministic and order-preserving (value a < value b implies
//     code a < code b);
//   * the sorted values stay on the device as the encode map, and a term
//     [lo, hi] becomes [min + L * step, min + (U - 1) * step] with
//     L = #{values < lo} and U = #{values <= hi} (empty when L >= U), found by
//     device binary searches for all terms of a call in one launch.  A scan
//     of the encoded table with rewritten terms selects exactly the rows the
//     original terms select on the original table.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "rts_internal.h"

namespace rts {
namespace {

__global__ void iota32_kernel(uint32_t *p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

__global__ void scatter_codes_kernel(const uint32_t *__restrict__ spos, uint64_t n, uint32_t emin, uint32_t step,
                                     uint32_t *__restrict__ codes) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x)
    codes[spos[r]] = emin + (uint32_t)r * step;
}

// out[i] = #{sval < key[i]} (lower bound) for each query key; a key of
// 2^32 (stored as has_key = 0) counts every value.
__global__ void lower_bound_kernel(const uint32_t *const *__restrict__ sval, const uint64_t n,
                                   const int32_t *__restrict__ col, const uint32_t *__restrict__ key,
                                   const uint8_t *__restrict__ has_key, int m, unsigned long long *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (!has_key[i]) {
    out[i] = n;
    return;
  }
  const uint32_t *s = sval[col[i]];
  uint64_t lo = 0, hi = n;
  const uint32_t k = key[i];
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (s[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  out[i] = lo;
}

template <class T>
T *dev_alloc(size_t count) {
  T *p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    throw Error(RTS_ERR_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
  }
  return p;
}

struct DevPtr {
  void *p = nullptr;
  ~DevPtr() {
    if (p) cudaFree(p);
  }
};

int grid_for(uint64_t n, int sm_count) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count * 8));
}

rts_status fail(rts_ctx *ctx, rts_status code, const char *what) {
  if (ctx) ctx->err = what;
  return set_thread_error(code, what);
}

}  // namespace

EncodeMap::~EncodeMap() {
  for (uint32_t *p : sval)
    if (p) cudaFree(p);
}

}  // namespace rts

extern "C" {

rts_status rts_encode_table(rts_ctx *ctx, uint32_t encode_min, uint32_t encode_max) {
  rts::Range nvtx_range_("rts_encode_table");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (ctx->cols.empty()) throw rts::Error(RTS_ERR_STATE, "no columns loaded");
    if (ctx->encode) throw rts::Error(RTS_ERR_STATE, "table is already encoded");
    const uint64_t n = ctx->nrows;
    if (n >= (1ull << 32)) throw rts::Error(RTS_ERR_ARG, "encoding supports fewer than 2^32 rows");
    if (encode_max <= encode_min || (uint64_t)(encode_max - encode_min) < n)
      throw rts::Error(RTS_ERR_ARG, "the code range must hold at least one code per row");
    const uint32_t step = (uint32_t)std::max<uint64_t>(1, ((uint64_t)encode_max - encode_min) / n);
    rts::DeviceGuard device_guard(ctx->device);
    const int nc = (int)ctx->cols.size();
    const uint64_t stride = (n + rts::kTileRows - 1) / rts::kTileRows * rts::kTileRows;
    auto map = std::make_unique<rts::EncodeMap>();
    map->n = n;
    map->min = encode_min;
    map->step = step;
    rts::DevPtr codes, ids, spos, temp;
    codes.p = rts::dev_alloc<uint32_t>((size_t)stride * nc);
    ids.p = rts::dev_alloc<uint32_t>(n);
    spos.p = rts::dev_alloc<uint32_t>(n);
    size_t temp_bytes = 0;
    RTS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                             (const uint32_t *)nullptr, (uint32_t *)nullptr, (int64_t)n, 0, 32));
    temp.p = rts::dev_alloc<char>(temp_bytes);
    RTS_CUDA(cudaMemset(codes.p, 0, (size_t)stride * nc * 4));
    for (int c = 0; c < nc; c++) {
      uint32_t *sv = rts::dev_alloc<uint32_t>(n);
      map->sval.push_back(sv);
      rts::iota32_kernel<<<rts::grid_for(n, ctx->sm_count), 256>>>((uint32_t *)ids.p, n);
      RTS_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, ctx->cols[c], sv, (const uint32_t *)ids.p,
                                               (uint32_t *)spos.p, (int64_t)n, 0, 32));
      rts::scatter_codes_kernel<<<rts::grid_for(n, ctx->sm_count), 256>>>(
          (const uint32_t *)spos.p, n, encode_min, step, (uint32_t *)codes.p + (size_t)stride * c);
    }
    RTS_CUDA(cudaGetLastError());
    RTS_CUDA(cudaDeviceSynchronize());
    // the codes replace the resident table (borrowed columns are left as they were)
    ctx->bindex.clear();
    ctx->bindex.resize(nc);
    if (ctx->owned) cudaFree(ctx->owned);
    ctx->owned = (uint32_t *)codes.p;
    ctx->owned_bytes = (size_t)stride * nc * 4;
    codes.p = nullptr;
    ctx->col_stride = stride;
    for (int c = 0; c < nc; c++) ctx->cols[c] = ctx->owned + (size_t)stride * c;
    ctx->encode = std::move(map);
    ctx->launches += 3 * nc;
    return RTS_OK;
  } catch (const rts::Error &e) {
    return rts::fail(ctx, e.code, e.what());
  } catch (const std::exception &e) {
    return rts::fail(ctx, RTS_ERR_NOMEM, e.what());
  }
}

rts_status rts_encode_terms(rts_ctx *ctx, const rts_term *terms, int32_t nterms, rts_term *out) {
  rts::Range nvtx_range_("rts_encode_terms");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  try {
    if (!ctx->encode) throw rts::Error(RTS_ERR_STATE, "table is not encoded (rts_encode_table)");
    if (nterms < 0 || (nterms > 0 && (!terms || !out))) throw rts::Error(RTS_ERR_ARG, "bad terms");
    if (nterms == 0) return RTS_OK;
    const rts::EncodeMap &E = *ctx->encode;
    const int nc = (int)E.sval.size();
    const int m = 2 * nterms;
    std::vector<int32_t> col(m);
    std::vector<uint32_t> key(m);
    std::vector<uint8_t> has(m);
    for (int i = 0; i < nterms; i++) {
      const rts_term &t = terms[i];
      if (t.column < 0 || t.column >= nc) throw rts::Error(RTS_ERR_ARG, "term column out of range");
      col[2 * i] = col[2 * i + 1] = t.column;
      key[2 * i] = t.lo;  // L = #{values < lo}
      has[2 * i] = 1;
      key[2 * i + 1] = t.hi + 1;  // U = #{values <= hi} = #{values < hi + 1}
      has[2 * i + 1] = t.hi != 0xFFFFFFFFu;
    }
    rts::DeviceGuard device_guard(ctx->device);
    const size_t bytes = (size_t)nc * 8 + (size_t)m * (4 + 4 + 1 + 8) + 64;
    rts::DevPtr buf;
    buf.p = rts::dev_alloc<char>(bytes);
    char *b = (char *)buf.p;
    auto *d_sval = (const uint32_t **)b;
    auto *d_out = (unsigned long long *)(b + (size_t)nc * 8);
    auto *d_col = (int32_t *)(b + (size_t)nc * 8 + (size_t)m * 8);
    auto *d_key = (uint32_t *)(b + (size_t)nc * 8 + (size_t)m * 12);
    auto *d_has = (uint8_t *)(b + (size_t)nc * 8 + (size_t)m * 16);
    RTS_CUDA(cudaMemcpy(d_sval, E.sval.data(), (size_t)nc * 8, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemcpy(d_col, col.data(), (size_t)m * 4, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemcpy(d_key, key.data(), (size_t)m * 4, cudaMemcpyHostToDevice));
    RTS_CUDA(cudaMemcpy(d_has, has.data(), (size_t)m, cudaMemcpyHostToDevice));
    rts::lower_bound_kernel<<<(m + 127) / 128, 128>>>(d_sval, E.n, d_col, d_key, d_has, m, d_out);
    RTS_CUDA(cudaGetLastError());
    std::vector<unsigned long long> rank(m);
    RTS_CUDA(cudaMemcpy(rank.data(), d_out, (size_t)m * 8, cudaMemcpyDeviceToHost));
    ctx->launches += 1;
    for (int i = 0; i < nterms; i++) {
      const uint64_t L = rank[2 * i], U = rank[2 * i + 1];
      out[i].column = terms[i].column;
      if (terms[i].lo > terms[i].hi || L >= U) {  // no value of the column lies in [lo, hi]
        out[i].lo = 1;
        out[i].hi = 0;
      } else {
        out[i].lo = E.min + (uint32_t)L * E.step;
        out[i].hi = E.min + (uint32_t)(U - 1) * E.step;
      }
    }
    return RTS_OK;
  } catch (const rts::Error &e) {
    return rts::fail(ctx, e.code, e.what());
  } catch (const std::exception &e) {
    return rts::fail(ctx, RTS_ERR_NOMEM, e.what());
  }
}

}  // extern "C"
