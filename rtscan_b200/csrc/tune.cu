// Autotuner for the batched kernel's launch shape.
//
// The batched kernel's speed depends on three knobs that trade shared memory
// against each other: warps per CTA (each warp stages 8 KB of result words),
// queries per pass (more queries share each row's interval lookups but need
// larger mask tables) and the mask-table budget (which fixes how many
// queries fit a pass and how many CTAs fit an SM).  rts_autotune_batch runs
// every candidate on a row sample of the resident table with the caller's
// queries, keeps the fastest, and can cache the choice in a small text file
// keyed by GPU, SM count, column count, table size and batch size.
//
// Candidates: variant 4 (pass shapes of 128/256/512 slots) with 16-warp
// CTAs at seven pass sizes from 128 to 512 queries and two table budgets,
// and with 8-warp CTAs (one per SM, or two when small tables leave room),
// and variant 3 at 8 and 16 warps per CTA with two budgets each.  The sample
// is the table's first rows: as many as the result bitmaps of the batch fit
// in a quarter of the free device memory, at least 2^24 and at most 2^27
// (all of a smaller table).  Each candidate runs once untimed and twice
// timed; the report (rts_autotune_report) lists every candidate's time.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "rts_internal.h"

namespace {

struct Candidate {
  int variant, warps, qpp;
  size_t budget;
};

std::vector<Candidate> candidates() {
  std::vector<Candidate> c;
  for (int qpp : {512, 448, 384, 320, 256, 192, 128})
    for (size_t budget : {(size_t)136 * 1024, (size_t)112 * 1024}) c.push_back({4, 16, qpp, budget});
  // 8-warp CTAs: one per SM with large tables, or two per SM when the
  // tables stay under about 56 KiB
  for (int qpp : {512, 256}) c.push_back({4, 8, qpp, (size_t)136 * 1024});
  for (int qpp : {512, 256, 128}) c.push_back({4, 8, qpp, (size_t)56 * 1024});
  for (size_t budget : {(size_t)88 * 1024, (size_t)64 * 1024}) c.push_back({3, 16, 256, budget});
  for (size_t budget : {(size_t)140 * 1024, (size_t)40 * 1024}) c.push_back({3, 8, 256, budget});
  return c;
}

size_t max_budget(int variant, int warps) {
  if (variant == 4) return 136 * 1024;
  return warps == 16 ? 88 * 1024 : 140 * 1024;
}

std::string cache_key(rts_ctx *ctx, int nq) {
  cudaDeviceProp p;
  std::string name = "gpu";
  if (cudaGetDeviceProperties(&p, ctx->device) == cudaSuccess) name = p.name;
  for (auto &ch : name)
    if (ch == ' ' || ch == '|') ch = '_';
  int lg = 0;
  while ((1ull << (lg + 1)) <= ctx->nrows) lg++;
  int qb = 1;
  while (qb < nq) qb <<= 1;
  return name + "|" + std::to_string(ctx->sm_count) + "|" + std::to_string(ctx->cols.size()) + "|" +
         std::to_string(lg) + "|" + std::to_string(qb);
}

bool cache_lookup(const char *path, const std::string &key, rts::BatchConfig *out) {
  if (!path) return false;
  FILE *f = fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool found = false;
  while (fgets(line, sizeof line, f)) {
    char k[400];
    int v, w, q;
    unsigned long b;
    double ms;
    if (sscanf(line, "%399s %d %d %d %lu %lf", k, &v, &w, &q, &b, &ms) == 6 && key == k) {
      out->variant = v;
      out->warps_per_cta = w;
      out->max_queries_per_pass = q;
      out->table_budget = b;
      found = true;
    }
  }
  fclose(f);
  return found;
}

void cache_store(const char *path, const std::string &key, const rts::BatchConfig &c, double ms) {
  if (!path) return;
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d %lu %.4f\n", key.c_str(), c.variant, c.warps_per_cta, c.max_queries_per_pass,
          (unsigned long)c.table_budget, ms);
  fclose(f);
}

bool valid(const rts_batch_config &c) {
  if (c.variant != 3 && c.variant != 4) return false;
  if (c.warps_per_cta != 8 && c.warps_per_cta != 16) return false;
  const int max_q = c.variant == 4 ? 512 : 256;
  return c.max_queries_per_pass >= 1 && c.max_queries_per_pass <= max_q && c.table_budget_bytes >= 4096 &&
         c.table_budget_bytes <= max_budget(c.variant, c.warps_per_cta);
}

}  // namespace

extern "C" {

rts_status rts_set_batch_config(rts_ctx *ctx, const rts_batch_config *cfg) {
  if (!ctx || !cfg) return rts::set_thread_error(RTS_ERR_ARG, "null argument");
  if (!valid(*cfg)) {
    ctx->err = "batch config out of range (variant 3|4, warps 8|16, queries per pass and table budget within "
               "the variant's limits)";
    return rts::set_thread_error(RTS_ERR_ARG, ctx->err);
  }
  ctx->batch_cfg.variant = cfg->variant;
  ctx->batch_cfg.warps_per_cta = cfg->warps_per_cta;
  ctx->batch_cfg.max_queries_per_pass = cfg->max_queries_per_pass;
  ctx->batch_cfg.table_budget = cfg->table_budget_bytes;
  return RTS_OK;
}

rts_status rts_get_batch_config(const rts_ctx *ctx, rts_batch_config *cfg) {
  if (!ctx || !cfg) return rts::set_thread_error(RTS_ERR_ARG, "null argument");
  cfg->variant = ctx->batch_cfg.variant;
  cfg->warps_per_cta = ctx->batch_cfg.warps_per_cta;
  cfg->max_queries_per_pass = ctx->batch_cfg.max_queries_per_pass;
  cfg->table_budget_bytes = (uint32_t)ctx->batch_cfg.table_budget;
  return RTS_OK;
}

rts_status rts_autotune_batch(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int32_t nq,
                              const char *cache_path, rts_batch_config *best_out) {
  rts::Range nvtx_range_("rts_autotune_batch");
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  if (ctx->cols.empty()) return rts::set_thread_error(RTS_ERR_STATE, "no columns loaded");
  if (nq < 1 || !offsets) return rts::set_thread_error(RTS_ERR_ARG, "need at least one query");
  const std::string key = cache_key(ctx, nq);
  rts::BatchConfig cached;
  if (cache_lookup(cache_path, key, &cached)) {
    ctx->batch_cfg = cached;
    ctx->tune_report = "{\"cached\": true}";
    if (best_out) rts_get_batch_config(ctx, best_out);
    return RTS_OK;
  }
  const uint64_t saved_n = ctx->nrows;
  const rts::BatchConfig saved_cfg = ctx->batch_cfg;
  uint32_t *bm = nullptr;
  unsigned long long *cnt = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  rts_status rc = RTS_OK;
  try {
    rts::DeviceGuard device_guard(ctx->device);
    // tune on the table's first rows: as many as a quarter of the free
    // memory holds the batch's bitmaps for, within [2^24, 2^27] rows
    size_t free_b = 0, total_b = 0;
    RTS_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const uint64_t fit = (uint64_t)((double)free_b / 4 / ((double)nq / 8)) & ~4095ull;
    const uint64_t sample = std::min<uint64_t>(saved_n, std::max<uint64_t>(1ull << 24, std::min<uint64_t>(fit, 1ull << 27)));
    ctx->nrows = sample;
    const uint64_t stride = (rts::words_for(sample) + 31) / 32 * 32;
    if (cudaMalloc(&bm, (size_t)nq * stride * 4) != cudaSuccess || cudaMalloc(&cnt, (size_t)nq * 8) != cudaSuccess) {
      cudaGetLastError();
      throw rts::Error(RTS_ERR_NOMEM, "autotune buffers do not fit");
    }
    RTS_CUDA(cudaEventCreate(&e0));
    RTS_CUDA(cudaEventCreate(&e1));
    double best_ms = 1e300;
    rts::BatchConfig best = saved_cfg;
    std::string report = "{\"sample_rows\": " + std::to_string(sample) + ", \"queries\": " + std::to_string(nq) +
                         ", \"candidates\": [";
    const rts::BatchConfig dflt;
    double default_ms = -1;
    bool first = true;
    for (const Candidate &c : candidates()) {
      ctx->batch_cfg.variant = c.variant;
      ctx->batch_cfg.warps_per_cta = c.warps;
      ctx->batch_cfg.max_queries_per_pass = c.qpp;
      ctx->batch_cfg.table_budget = c.budget;
      rts::batch_scan(ctx, terms, offsets, nq, bm, stride, cnt, nullptr, c.budget);  // warm-up
      RTS_CUDA(cudaEventRecord(e0, nullptr));
      for (int r = 0; r < 2; r++) rts::batch_scan(ctx, terms, offsets, nq, bm, stride, cnt, nullptr, c.budget);
      RTS_CUDA(cudaEventRecord(e1, nullptr));
      RTS_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      RTS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      char item[160];
      snprintf(item, sizeof item, "%s{\"variant\": %d, \"warps_per_cta\": %d, \"max_queries_per_pass\": %d, "
               "\"table_budget_bytes\": %zu, \"ms\": %.4f}", first ? "" : ", ", c.variant, c.warps, c.qpp, c.budget,
               ms / 2);
      report += item;
      first = false;
      if (c.variant == dflt.variant && c.warps == dflt.warps_per_cta && c.qpp == dflt.max_queries_per_pass &&
          c.budget == dflt.table_budget)
        default_ms = ms / 2;
      if (ms / 2 < best_ms) {
        best_ms = ms / 2;
        best = ctx->batch_cfg;
      }
    }
    char tail[160];
    snprintf(tail, sizeof tail, "], \"best_ms\": %.4f, \"default_ms\": %.4f}", best_ms, default_ms);
    ctx->tune_report = report + tail;
    ctx->batch_cfg = best;
    ctx->nrows = saved_n;
    cache_store(cache_path, key, best, best_ms);
  } catch (const std::exception &e) {
    ctx->nrows = saved_n;
    ctx->batch_cfg = saved_cfg;
    ctx->err = e.what();
    rc = rts::set_thread_error(rts::status_of(e), e.what());
  }
  if (bm) cudaFree(bm);
  if (cnt) cudaFree(cnt);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (rc == RTS_OK && best_out) rts_get_batch_config(ctx, best_out);
  return rc;
}

rts_status rts_autotune_report(const rts_ctx *ctx, char *buf, uint64_t size, uint64_t *needed) {
  if (!ctx) return rts::set_thread_error(RTS_ERR_ARG, "null context");
  const std::string &r = ctx->tune_report;
  if (needed) *needed = r.size() + 1;
  if (buf && size) {
    const size_t m = std::min<size_t>(r.size(), size - 1);
    memcpy(buf, r.data(), m);
    buf[m] = '\0';
  }
  return RTS_OK;
}

}  // extern "C"
