// Prepared batches: a batch planned once and replayed as a CUDA graph.
//
// A caller that answers the same batch of queries again and again (a
// dashboard refresh, a standing query set over a table that is reloaded in
// place) prepares it once: the host plans the passes, uploads the mask
// tables, and captures every launch of the batch -- count reset, fill and
// fused launches for the queries outside the batched kernel, the shared
// position search when the batch has several passes, one batched kernel per
// pass -- into a CUDA graph.  Each rts_batch_launch is then one
// cudaGraphLaunch: no host planning and no per-kernel launch overhead.  The
// graph reads the context's resident columns at the addresses they had when
// it was prepared, so it must be re-prepared after the table is reloaded.
#include <cuda_runtime.h>

#include <vector>

#include "batch_plan.h"
#include "rts_internal.h"

struct rts_prepared {
  rts_ctx *ctx = nullptr;
  uint32_t *blob = nullptr;
  void *scratch = nullptr;  // the batch's shared positions (its own: the graph keeps the address)
  size_t scratch_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;  // kernels launched per replay
  ~rts_prepared() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (blob) cudaFree(blob);
    if (scratch) cudaFree(scratch);
  }
};

namespace {
rts_status fail(rts_ctx *ctx, rts_status code, const std::string &m) {
  if (ctx) ctx->err = m;
  return rts::set_thread_error(code, m);
}
}  // namespace

extern "C" {

rts_status rts_batch_prepare(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int32_t nq,
                             uint32_t *dev_bitmaps, uint64_t stride_words, uint64_t *dev_counts, rts_prepared **out) {
  rts::Range nvtx_range_("rts_batch_prepare");
  if (!ctx || !out) return rts::set_thread_error(RTS_ERR_ARG, "null argument");
  *out = nullptr;
  if (ctx->cols.empty()) return fail(ctx, RTS_ERR_STATE, "no columns loaded");
  if (nq < 1 || !offsets || !dev_bitmaps || !dev_counts) return fail(ctx, RTS_ERR_ARG, "bad batch arguments");
  if (stride_words < rts::words_for(ctx->nrows)) return fail(ctx, RTS_ERR_ARG, "stride_words smaller than a bitmap");
  auto *p = new rts_prepared();
  p->ctx = ctx;
  cudaStream_t cap = nullptr;
  try {
    rts::DeviceGuard device_guard(ctx->device);
    std::vector<rts::NormQuery> norm = rts::normalize_all(ctx, terms, offsets, nq);
    std::vector<int> inside, outside;
    for (int q = 0; q < nq; q++) (rts::runs_in_kernel(norm[q]) ? inside : outside).push_back(q);
    rts::BatchPlanPtr plan;
    if (!inside.empty()) {
      plan = rts::make_batch_plan(ctx, norm, inside, nullptr, ctx->batch_cfg.table_budget, true);
      const auto &blob = rts::batch_plan_blob(*plan);
      if (cudaMalloc(&p->blob, std::max<size_t>(blob.size(), 4) * 4) != cudaSuccess) {
        cudaGetLastError();
        throw rts::Error(RTS_ERR_NOMEM, "plan allocation failed");
      }
      RTS_CUDA(cudaMemcpy(p->blob, blob.data(), blob.size() * 4, cudaMemcpyHostToDevice));
      // shared positions when there is room (at most an eighth of the device);
      // without them every pass searches its own
      const size_t need = rts::batch_plan_scratch_bytes(*plan, ctx->nrows);
      size_t free_b = 0, total_b = 0;
      if (need && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need <= total_b / 8 &&
          cudaMalloc(&p->scratch, need) == cudaSuccess)
        p->scratch_bytes = need;
      cudaGetLastError();
    }
    unsigned long long *counts = reinterpret_cast<unsigned long long *>(dev_counts);
    RTS_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    auto record = [&](cudaStream_t s) {
      uint64_t k = 0;
      RTS_CUDA(cudaMemsetAsync(counts, 0, (size_t)nq * 8, s));
      k += rts::launch_outside(ctx, norm, outside, nullptr, dev_bitmaps, stride_words, counts, s);
      if (plan)
        k += rts::launch_batch_plan(ctx, *plan, p->blob, dev_bitmaps, stride_words, counts, 0, ctx->nrows, p->scratch,
                                    p->scratch_bytes, s);
      return k;
    };
    // one uncaptured run sets up launch attributes and checks the launches
    p->kernels = record(cap);
    RTS_CUDA(cudaStreamSynchronize(cap));
    RTS_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    try {
      record(cap);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(cap, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    RTS_CUDA(cudaStreamEndCapture(cap, &p->graph));
    RTS_CUDA(cudaGraphInstantiate(&p->exec, p->graph, 0));
    cudaStreamDestroy(cap);
    ctx->launches += p->kernels;
    *out = p;
    return RTS_OK;
  } catch (const std::exception &e) {
    if (cap) cudaStreamDestroy(cap);
    delete p;
    return fail(ctx, rts::status_of(e), e.what());
  }
}

rts_status rts_batch_launch(rts_prepared *p, void *stream) {
  rts::Range nvtx_range_("rts_batch_launch");
  if (!p) return rts::set_thread_error(RTS_ERR_ARG, "null prepared batch");
  cudaError_t e = cudaGraphLaunch(p->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    try {
      return fail(p->ctx, RTS_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
    } catch (const std::exception &) {  // no room for the message
      return RTS_ERR_CUDA;
    }
  }
  p->ctx->launches += p->kernels;
  return RTS_OK;
}

void rts_batch_release(rts_prepared *p) { delete p; }

}  // extern "C"
