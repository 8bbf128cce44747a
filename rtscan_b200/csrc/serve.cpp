// Continuous-batching scan server (rts_server_*).
//
// The reference has no serving path: its drivers read a query, scan, check
// and print, one at a time (bindex_cuda.cpp:1827-1986).  The server keeps
// the context's columns resident and answers a stream of requests with the
// batched kernel, as a circular shared scan:
//
//   * Memory admission: a pool of `max_active` result slots (one bitmap and
//     one count each) bounds the requests on the GPU; requests wait in a
//     bounded queue (RTS_ERR_FULL beyond it) until a slot is free.
//   * The table is cut into segments of `segment_rows` rows.  Each step
//     runs the batched kernel over one segment for every active request and
//     then moves a cursor to the next segment, wrapping around.  A request
//     admitted while the cursor is at segment c0 has seen every segment once
//     when it has been in the scan for one segment of each; its count,
//     accumulated per segment, and its bitmap are then final.  New arrivals
//     join at the next plan, so their work overlaps on the device with
//     requests already running.
//   * The worker thread plans the active set (mask tables) when requests
//     arrive, at most every kReplanSteps steps while the running plan still
//     has requests, keeps at most `max_inflight_steps` steps queued on its
//     stream, and marks a request done when the event recorded after its
//     last step has completed.  A request that finishes or is cancelled
//     leaves the running plan without a re-plan: its slot entries in the
//     plan become -1 (one small launch per step), which every batch kernel
//     skips.  Planning and the plan upload (which waits for the steps still
//     reading the other plan buffer) run without the server lock, so
//     submitters and pollers never wait behind them; the lock covers
//     admission, the step's launches and the bookkeeping only.
//   * The requests finishing at a step share one copy of their counts to
//     pinned host memory and one event, queued right after the step, so
//     poll/wait/fetch read a count without touching the device; a bitmap
//     fetch copies outside the lock.
// Requests the batched kernel does not take (an empty term, no constrained
// column, more than eight columns) are answered in one launch at admission.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_plan.h"
#include "rts_internal.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// FREE -> ACTIVE (scanning) -> FINISHING (last step queued) -> DONE ->
// FETCHING (a bitmap copy in progress) -> FREE; ACTIVE/FINISHING ->
// CANCELLING -> FREE once the steps queued before the cancel are done.
enum SlotState { FREE = 0, ACTIVE, FINISHING, DONE, CANCELLING, FETCHING };

struct Request {
  uint64_t ticket;
  std::vector<rts_term> terms;
  double t_submit;
};

}  // namespace

struct rts_server {
  rts_ctx *ctx = nullptr;
  rts_server_config cfg{};
  uint64_t nrows = 0, words = 0, stride = 0, seg_rows = 0;
  int nseg = 0;
  uint32_t *bitmaps = nullptr;
  unsigned long long *counts = nullptr;
  void *pre = nullptr;  // a segment's shared positions (null: every pass searches)
  size_t pre_bytes = 0;
  unsigned long long *host_counts = nullptr;  // pinned; slot i's count once it is DONE
  cudaStream_t stream = nullptr, copy_stream = nullptr;

  struct PlanBuf {
    uint32_t *dev = nullptr;
    size_t cap = 0;
    uint32_t *host = nullptr;
    size_t hcap = 0;
    cudaEvent_t done = nullptr;
  } pb[2];
  int next_pb = 0;

  struct Slot {
    SlotState state = FREE;
    uint64_t ticket = 0;
    rts::NormQuery q;
    int start_seg = 0, segs_done = 0;
    double t_submit = 0, t_done = 0;
    cudaEvent_t ev = nullptr;
    uint64_t count = 0;
  };
  std::vector<Slot> slots;
  std::vector<int> free_slots;
  std::unordered_map<uint64_t, int> ticket_slot;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request> queue;
  uint64_t next_ticket = 1;
  int cursor = 0;
  uint64_t active_version = 1, plan_version = 0;
  uint64_t plan_step = 0;                // steps launched when the running plan was made
  double last_plan_s = 0;                // host time of the last plan and upload
  double step_s = 0;                     // moving average of the GPU's time per step
  double last_retire = 0;
  static constexpr uint64_t kReplanSteps = 2;
  rts::BatchPlanPtr plan;
  const uint32_t *plan_dev = nullptr;
  std::vector<int> plan_slots;
  std::deque<cudaEvent_t> inflight;
  std::vector<cudaEvent_t> event_pool;

  // statistics
  uint64_t submitted = 0, completed = 0, rejected = 0, cancelled = 0, steps = 0, plans = 0;
  double plan_s = 0;  // host time of the plans and their uploads
  std::vector<double> latencies;
  std::string fatal;
  // completions (ticket, done time) for a running replay
  bool track_done = false;
  std::vector<std::pair<uint64_t, double>> done_tickets;

  std::atomic<bool> stop{false};
  std::thread worker;

  // Events that slots wait on, with the number of slots waiting on each
  // (the requests finishing at one step share one event).
  std::unordered_map<cudaEvent_t, int> ev_refs;
  void hold(cudaEvent_t e) { ev_refs[e]++; }
  void drop(cudaEvent_t e) {
    auto it = ev_refs.find(e);
    if (it != ev_refs.end() && --it->second == 0) {
      ev_refs.erase(it);
      put_event(e);
    }
  }

  cudaEvent_t get_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    RTS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return e;
  }
  void put_event(cudaEvent_t e) { event_pool.push_back(e); }

  // Copy a plan blob into the plan buffer not used by the previous plan,
  // after the steps that still read it (worker thread, lock not held).
  void upload(const std::vector<uint32_t> &blob) {
    PlanBuf &b = pb[next_pb];
    next_pb ^= 1;
    const size_t bytes = std::max<size_t>(blob.size(), 4) * 4;
    if (b.done) RTS_CUDA(cudaEventSynchronize(b.done));
    else RTS_CUDA(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    if (b.cap < bytes) {
      if (b.dev) cudaFree(b.dev);
      b.dev = nullptr;
      b.cap = 0;
      if (cudaMalloc(&b.dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw rts::Error(RTS_ERR_NOMEM, "server plan allocation failed");
      }
      b.cap = bytes;
    }
    if (b.hcap < bytes) {
      if (b.host) cudaFreeHost(b.host);
      b.host = nullptr;
      RTS_CUDA(cudaMallocHost(&b.host, bytes));
      b.hcap = bytes;
    }
    memcpy(b.host, blob.data(), blob.size() * 4);
    RTS_CUDA(cudaMemcpyAsync(b.dev, b.host, blob.size() * 4, cudaMemcpyHostToDevice, stream));
    plan_dev = b.dev;
    // record the buffer's release after the steps that use it: done at the
    // next upload into the other buffer, recorded below after each step
    current_pb = &b;
  }
  PlanBuf *current_pb = nullptr;

  // Admit queued requests into free slots (mu held); their counts are
  // zeroed by one launch.
  void admit() {
    std::vector<int32_t> fresh;
    while (!queue.empty() && !free_slots.empty()) {
      Request r = std::move(queue.front());
      queue.pop_front();
      const int sl = free_slots.back();
      free_slots.pop_back();
      Slot &S = slots[sl];
      S.q = rts::normalize(r.terms.data(), (int)r.terms.size(), sl, (int)ctx->cols.size());
      S.ticket = r.ticket;
      S.t_submit = r.t_submit;
      S.segs_done = 0;
      S.start_seg = cursor;
      S.count = 0;
      ticket_slot[r.ticket] = sl;
      if (!rts::runs_in_kernel(S.q)) {
        std::vector<rts::NormQuery> one(slots.size());
        one[sl] = S.q;
        ctx->launches += rts::launch_outside(ctx, one, {sl}, nullptr, bitmaps, stride, counts, stream);
        finish(sl);
      } else {
        fresh.push_back(sl);
        S.state = ACTIVE;
        active_version++;
      }
    }
    if (!fresh.empty()) {
      rts::launch_zero_counts(counts, fresh.data(), (int)fresh.size(), stream);
      ctx->launches += ((int)fresh.size() + 511) / 512;
    }
  }

  // Queue the copy of slot sl's count to the host and the event that marks
  // the slot done, behind every launch that writes it (mu held).
  void finish(int sl) { finish_all(&sl, 1); }

  // The same for the slots finishing at one step: one copy of the counts
  // from the lowest to the highest of them (the others' device counts are
  // unchanged or not yet read) and one event they share (mu held).
  void finish_all(const int *sl, int n) {
    if (n == 0) return;
    const int lo = *std::min_element(sl, sl + n), hi = *std::max_element(sl, sl + n);
    RTS_CUDA(cudaMemcpyAsync(host_counts + lo, counts + lo, (size_t)(hi - lo + 1) * 8, cudaMemcpyDeviceToHost,
                             stream));
    cudaEvent_t e = get_event();
    RTS_CUDA(cudaEventRecord(e, stream));
    for (int i = 0; i < n; i++) {
      Slot &S = slots[sl[i]];
      S.ev = e;
      hold(e);
      S.state = FINISHING;
    }
  }

  // Slots cancelled while active get their release event here, after every
  // launch queued so far, some of which may still write them (mu held).
  void fence_cancels() {
    std::vector<int> gone;
    for (size_t i = 0; i < slots.size(); i++)
      if (slots[i].state == CANCELLING && !slots[i].ev) gone.push_back((int)i);
    if (gone.empty()) return;
    unplan(gone);  // no later step writes them
    for (int sl : gone) {
      Slot &S = slots[sl];
      S.ev = get_event();
      hold(S.ev);
      RTS_CUDA(cudaEventRecord(S.ev, stream));
    }
  }

  // Take slots out of the running plan (mu held): their entries in the
  // plan's slot maps become -1 (on the device by one launch, queued before
  // the next step), and the steps stop counting segments for them.
  void unplan(const std::vector<int> &gone) {
    if (!plan || gone.empty()) return;
    std::vector<uint32_t> words;
    for (int sl : gone) rts::batch_plan_drop(*plan, sl, words);
    if (!words.empty()) {
      rts::launch_set_words(const_cast<uint32_t *>(plan_dev), words.data(), (int)words.size(), 0xFFFFFFFFu, stream);
      ctx->launches += ((int)words.size() + 511) / 512;
    }
    plan_slots.erase(std::remove_if(plan_slots.begin(), plan_slots.end(),
                                    [&](int sl) { return std::find(gone.begin(), gone.end(), sl) != gone.end(); }),
                     plan_slots.end());
  }

  // The active set, and a copy of its queries when it differs from the
  // planned one (mu held): -1 nothing is active, 0 the plan is current, 1
  // `norm` holds the queries to plan.  Only the worker admits and retires
  // requests, so until the step is launched the set can lose cancelled
  // slots only.
  int snapshot(std::vector<int> &active, std::vector<rts::NormQuery> &norm, uint64_t &version) {
    active.clear();
    for (size_t i = 0; i < slots.size(); i++)
      if (slots[i].state == ACTIVE) active.push_back((int)i);
    if (active.empty()) return -1;
    if (plan_version == active_version) return 0;
    // New arrivals join at the next plan.  When planning takes the host
    // longer than the GPU takes for a step (a slow host, a large active
    // set), plans are made at most every kReplanSteps steps while the
    // running plan still has requests: between plans the worker launches
    // steps back to back, so the GPU runs the steps queued during a plan's
    // host work.  Otherwise every change is planned at once (a deferred plan
    // carries its finished requests' slots one step longer).
    if (plan && !plan_slots.empty() && steps - plan_step < kReplanSteps && last_plan_s > step_s) return 0;
    norm.assign(slots.size(), rts::NormQuery());
    for (int sl : active) norm[sl] = slots[sl].q;
    version = active_version;
    return 1;
  }

  // Launch one step of the current plan over the segment at the cursor and
  // retire the requests that have now seen every segment (mu held).
  void step() {
    rts::Range nvtx_range_("rts_server_step");
    if (!plan || plan_slots.empty()) return;
    const uint64_t r0 = (uint64_t)cursor * seg_rows;
    const uint64_t r1 = std::min<uint64_t>(nrows, r0 + seg_rows);
    // the segment's shared positions, when the plan has them, in the
    // server's scratch (steps run one after another on the stream)
    ctx->launches += rts::launch_batch_plan(ctx, *plan, plan_dev, bitmaps, stride, counts, r0, r1, pre, pre_bytes,
                                            stream);
    RTS_CUDA(cudaGetLastError());
    cudaEvent_t ev = get_event();
    RTS_CUDA(cudaEventRecord(ev, stream));
    inflight.push_back(ev);
    if (current_pb) RTS_CUDA(cudaEventRecord(current_pb->done, stream));
    steps++;
    cursor = (cursor + 1) % nseg;
    std::vector<int> done_now;
    for (int sl : plan_slots) {
      Slot &S = slots[sl];
      if (S.state != ACTIVE) continue;  // cancelled since the plan was made
      if (++S.segs_done == nseg) done_now.push_back(sl);
    }
    finish_all(done_now.data(), (int)done_now.size());
    // the plan keeps running without them; when planning is cheaper than a
    // step, the next step gets a plan without their slots as well
    unplan(done_now);
    if (!done_now.empty() && last_plan_s <= step_s) active_version++;
  }

  // Mark finished requests done (mu held).
  void reap() {
    bool any = false;
    std::unordered_map<cudaEvent_t, cudaError_t> state;  // each shared event queried once
    for (size_t i = 0; i < slots.size(); i++) {
      Slot &S = slots[i];
      if (S.state != FINISHING && S.state != CANCELLING) continue;
      if (!S.ev) continue;  // a cancel not fenced yet
      auto st = state.find(S.ev);
      if (st == state.end()) st = state.emplace(S.ev, cudaEventQuery(S.ev)).first;
      const cudaError_t e = st->second;
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) throw rts::Error(RTS_ERR_CUDA, std::string("server step: ") + cudaGetErrorString(e));
      drop(S.ev);
      S.ev = nullptr;
      if (S.state == CANCELLING) {
        S.state = FREE;
        free_slots.push_back((int)i);
        continue;
      }
      S.state = DONE;
      S.t_done = now_s();
      latencies.push_back(S.t_done - S.t_submit);
      completed++;
      if (track_done) done_tickets.emplace_back(S.ticket, S.t_done);
      any = true;
    }
    if (any) cv_done.notify_all();
  }

  void run() {
    cudaSetDevice(ctx->device);
    try {
      std::vector<int> active;
      std::vector<rts::NormQuery> norm;
      while (!stop.load()) {
        // bound the steps queued on the stream, without holding the lock
        std::vector<cudaEvent_t> retired;
        while ((int)inflight.size() >= cfg.max_inflight_steps) {
          // a step still running when the worker comes for it: the GPU, not
          // the host, sets the pace, and the interval between two such
          // finished steps is the GPU's time per step
          const bool gpu_paced = cudaEventQuery(inflight.front()) == cudaErrorNotReady;
          RTS_CUDA(cudaEventSynchronize(inflight.front()));
          retired.push_back(inflight.front());
          inflight.pop_front();
          const double t = now_s();
          if (gpu_paced && last_retire > 0)
            step_s = step_s > 0 ? 0.9 * step_s + 0.1 * (t - last_retire) : t - last_retire;
          last_retire = gpu_paced ? t : 0;
        }
        uint64_t version = 0;
        int todo = -1;
        {
          std::unique_lock<std::mutex> lk(mu);
          for (auto e : retired) put_event(e);
          admit();
          fence_cancels();
          reap();
          bool busy = false;
          for (auto &S : slots)
            if (S.state == ACTIVE || S.state == FINISHING || S.state == CANCELLING) busy = true;
          if (!busy && queue.empty()) {
            last_retire = 0;  // idle time is no step time
            cv_work.wait_for(lk, std::chrono::milliseconds(2));
            continue;
          }
          todo = snapshot(active, norm, version);
          if (todo < 0) {  // only finishing or cancelled requests: wait for their events
            fence_cancels();
            cv_work.wait_for(lk, std::chrono::microseconds(200));
            continue;
          }
        }
        if (todo == 1) {  // plan and upload without the lock
          const double t0 = now_s();
          rts::BatchPlanPtr p = rts::make_batch_plan(ctx, norm, active, nullptr, ctx->batch_cfg.table_budget, true);
          upload(rts::batch_plan_blob(*p));
          const double t1 = now_s();
          std::lock_guard<std::mutex> lk(mu);
          plans++;
          plan_s += t1 - t0;
          last_plan_s = t1 - t0;
          plan = std::move(p);
          plan_slots = active;
          plan_version = version;
          plan_step = steps;
          // requests cancelled while it was planned run no step of it
          std::vector<int> gone;
          for (int sl : active)
            if (slots[sl].state != ACTIVE) gone.push_back(sl);
          unplan(gone);
        }
        {
          std::lock_guard<std::mutex> lk(mu);
          step();
          fence_cancels();
        }
        // let clients in between steps
        std::this_thread::yield();
      }
    } catch (const std::exception &e) {
      std::lock_guard<std::mutex> lk(mu);
      fatal = e.what();
      cv_done.notify_all();
    }
  }

  ~rts_server() {
    stop.store(true);
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
    // runs on the caller's thread (rts_server_stop, or a failed start):
    // switch to the context's device and give the caller's back at the end
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(ctx->device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto &b : pb) {
      if (b.dev) cudaFree(b.dev);
      if (b.host) cudaFreeHost(b.host);
      if (b.done) cudaEventDestroy(b.done);
    }
    for (auto e : inflight) cudaEventDestroy(e);
    for (auto e : event_pool) cudaEventDestroy(e);
    for (auto &kv : ev_refs) cudaEventDestroy(kv.first);  // each slot event once
    if (bitmaps) cudaFree(bitmaps);
    if (counts) cudaFree(counts);
    if (pre) cudaFree(pre);
    if (host_counts) cudaFreeHost(host_counts);
    if (stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  }
};

namespace {

rts_status fail(rts_server *srv, rts_status code, const std::string &m) {
  if (srv && srv->ctx) srv->ctx->err = m;
  return rts::set_thread_error(code, m);
}

// Run a C-ABI body and turn an exception (a host allocation that failed, a
// thread that could not start) into a status, so that none crosses the C
// boundary.
template <class F>
rts_status srv_guarded(rts_server *srv, F &&f) {
  try {
    return f();
  } catch (const rts::Error &e) {
    return fail(srv, e.code, e.what());
  } catch (const std::bad_alloc &) {
    return fail(srv, RTS_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(srv, RTS_ERR_STATE, e.what());
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double idx = p * (double)(v.size() - 1);
  const size_t lo = (size_t)idx, hi = std::min(v.size() - 1, lo + 1);
  return v[lo] + (v[hi] - v[lo]) * (idx - (double)lo);
}

}  // namespace

extern "C" {

rts_status rts_server_start(rts_ctx *ctx, const rts_server_config *cfg, rts_server **out) {
  if (!ctx || !out) return rts::set_thread_error(RTS_ERR_ARG, "null argument");
  *out = nullptr;
  if (ctx->cols.empty()) return rts::set_thread_error(RTS_ERR_STATE, "no columns loaded");
  auto *srv = new rts_server();
  try {
    srv->ctx = ctx;
    rts_server_config c{};
    c.max_active = 512;
    c.max_queue = 1 << 16;
    c.segment_rows = 1ull << 22;
    c.max_inflight_steps = 3;
    if (cfg) {
      if (cfg->max_active > 0) c.max_active = cfg->max_active;
      if (cfg->max_queue > 0) c.max_queue = cfg->max_queue;
      if (cfg->segment_rows > 0) c.segment_rows = cfg->segment_rows;
      if (cfg->max_inflight_steps > 0) c.max_inflight_steps = cfg->max_inflight_steps;
    }
    if (c.segment_rows % 4096) throw rts::Error(RTS_ERR_ARG, "segment_rows must be a multiple of 4096");
    srv->cfg = c;
    rts::DeviceGuard device_guard(ctx->device);
    srv->nrows = ctx->nrows;
    srv->words = rts::words_for(ctx->nrows);
    srv->stride = (srv->words + 31) / 32 * 32;
    srv->seg_rows = c.segment_rows;
    srv->nseg = (int)((srv->nrows + c.segment_rows - 1) / c.segment_rows);
    const size_t bm_bytes = (size_t)c.max_active * srv->stride * 4;
    if (cudaMalloc(&srv->bitmaps, bm_bytes) != cudaSuccess || cudaMalloc(&srv->counts, (size_t)c.max_active * 8) != cudaSuccess) {
      cudaGetLastError();
      throw rts::Error(RTS_ERR_NOMEM, "result pool of " + std::to_string(bm_bytes) + " bytes does not fit");
    }
    RTS_CUDA(cudaMallocHost(&srv->host_counts, (size_t)c.max_active * 8));
    // shared positions of one segment, 8 bytes per row and sharing pass
    // (268 MB for 2^23-row segments); without it every pass searches
    srv->pre_bytes = rts::kMaxSharedPasses * (size_t)(c.segment_rows + 2) * 8;
    if (cudaMalloc(&srv->pre, srv->pre_bytes) != cudaSuccess) {
      cudaGetLastError();
      srv->pre = nullptr;
      srv->pre_bytes = 0;
    }
    RTS_CUDA(cudaStreamCreateWithFlags(&srv->stream, cudaStreamNonBlocking));
    RTS_CUDA(cudaStreamCreateWithFlags(&srv->copy_stream, cudaStreamNonBlocking));
    srv->slots.resize(c.max_active);
    for (int i = c.max_active - 1; i >= 0; i--) srv->free_slots.push_back(i);
    srv->worker = std::thread([srv] { srv->run(); });
    *out = srv;
    return RTS_OK;
  } catch (const std::exception &e) {
    delete srv;
    ctx->err = e.what();
    return rts::set_thread_error(rts::status_of(e), e.what());
  }
}

rts_status rts_server_submit(rts_server *srv, const rts_term *terms, int32_t nterms, uint64_t *ticket) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv || !ticket || nterms < 0 || (nterms > 0 && !terms)) return fail(srv, RTS_ERR_ARG, "bad submit arguments");
    for (int i = 0; i < nterms; i++)
      if (terms[i].column < 0 || terms[i].column >= (int)srv->ctx->cols.size())
        return fail(srv, RTS_ERR_ARG, "term column out of range");
    const double t_submit = now_s();
    std::lock_guard<std::mutex> lk(srv->mu);
    if (!srv->fatal.empty()) return fail(srv, RTS_ERR_CUDA, "server stopped: " + srv->fatal);
    if ((int64_t)srv->queue.size() >= srv->cfg.max_queue) {
      srv->rejected++;
      return fail(srv, RTS_ERR_FULL, "request queue full");
    }
    Request r;
    r.ticket = srv->next_ticket++;
    r.terms.assign(terms, terms + nterms);
    r.t_submit = t_submit;
    *ticket = r.ticket;
    srv->queue.push_back(std::move(r));
    srv->submitted++;
    srv->cv_work.notify_one();
    return RTS_OK;
  });
}

rts_status rts_server_poll(rts_server *srv, uint64_t ticket, int32_t *done, uint64_t *count) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv || !done) return fail(srv, RTS_ERR_ARG, "bad poll arguments");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (!srv->fatal.empty()) return fail(srv, RTS_ERR_CUDA, "server stopped: " + srv->fatal);
    *done = 0;
    auto it = srv->ticket_slot.find(ticket);
    if (it == srv->ticket_slot.end()) {
      for (auto &r : srv->queue)
        if (r.ticket == ticket) return RTS_OK;
      return fail(srv, RTS_ERR_ARG, "unknown ticket");
    }
    rts_server::Slot &S = srv->slots[it->second];
    if (S.state == DONE || S.state == FETCHING) {
      *done = 1;
      if (count) *count = srv->host_counts[it->second];
    }
    return RTS_OK;
  });
}

rts_status rts_server_wait(rts_server *srv, uint64_t ticket, int32_t timeout_ms, uint64_t *count) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv) return fail(srv, RTS_ERR_ARG, "null server");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
    std::unique_lock<std::mutex> lk(srv->mu);
    while (true) {
      if (!srv->fatal.empty()) return fail(srv, RTS_ERR_CUDA, "server stopped: " + srv->fatal);
      auto it = srv->ticket_slot.find(ticket);
      if (it != srv->ticket_slot.end() &&
          (srv->slots[it->second].state == DONE || srv->slots[it->second].state == FETCHING)) {
        if (count) *count = srv->host_counts[it->second];
        return RTS_OK;
      }
      if (it == srv->ticket_slot.end()) {
        bool queued = false;
        for (auto &r : srv->queue) queued = queued || r.ticket == ticket;
        if (!queued) return fail(srv, RTS_ERR_ARG, "unknown ticket");
      }
      if (srv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
        auto it2 = srv->ticket_slot.find(ticket);
        if (it2 != srv->ticket_slot.end() &&
            (srv->slots[it2->second].state == DONE || srv->slots[it2->second].state == FETCHING))
          continue;
        return fail(srv, RTS_ERR_TIMEOUT, "request not done within the timeout");
      }
    }
  });
}

rts_status rts_server_fetch(rts_server *srv, uint64_t ticket, uint32_t *host_bitmap, uint64_t *count) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv) return fail(srv, RTS_ERR_ARG, "null server");
    int sl;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      auto it = srv->ticket_slot.find(ticket);
      if (it == srv->ticket_slot.end()) return fail(srv, RTS_ERR_ARG, "unknown or unfinished ticket");
      sl = it->second;
      rts_server::Slot &S = srv->slots[sl];
      if (S.state == FETCHING) return fail(srv, RTS_ERR_STATE, "request is being fetched by another call");
      if (S.state != DONE) return fail(srv, RTS_ERR_STATE, "request not done");
      if (count) *count = srv->host_counts[sl];
      if (!host_bitmap) {  // the count is already on the host: release the slot
        S.state = FREE;
        srv->ticket_slot.erase(it);
        srv->free_slots.push_back(sl);
        srv->cv_work.notify_one();
        return RTS_OK;
      }
      S.state = FETCHING;  // nobody frees or reuses the slot during the copy
    }
    // the bitmap leaves without the lock held
    rts::DeviceGuard device_guard(srv->ctx->device);
    cudaError_t e = cudaMemcpyAsync(host_bitmap, srv->bitmaps + (uint64_t)sl * srv->stride, srv->words * 4,
                                    cudaMemcpyDeviceToHost, srv->copy_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(srv->copy_stream);
    std::lock_guard<std::mutex> lk(srv->mu);
    rts_server::Slot &S = srv->slots[sl];
    if (e != cudaSuccess) {
      S.state = DONE;  // the caller may try again
      return fail(srv, RTS_ERR_CUDA, std::string("fetch: ") + cudaGetErrorString(e));
    }
    S.state = FREE;
    srv->ticket_slot.erase(ticket);
    srv->free_slots.push_back(sl);
    srv->cv_work.notify_one();
    return RTS_OK;
  });
}

rts_status rts_server_cancel(rts_server *srv, uint64_t ticket) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv) return fail(srv, RTS_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(srv->mu);
    for (auto it = srv->queue.begin(); it != srv->queue.end(); ++it)
      if (it->ticket == ticket) {
        srv->queue.erase(it);
        srv->cancelled++;
        return RTS_OK;
      }
    auto it = srv->ticket_slot.find(ticket);
    if (it == srv->ticket_slot.end()) return fail(srv, RTS_ERR_ARG, "unknown ticket");
    rts_server::Slot &S = srv->slots[it->second];
    if (S.state == FETCHING) return fail(srv, RTS_ERR_STATE, "request is being fetched");
    if (S.state == ACTIVE) {
      // kernels already queued (or being queued by the worker) may still
      // write this slot: the worker records its release event after them
      S.state = CANCELLING;
      srv->active_version++;
      srv->cv_work.notify_one();
    } else if (S.state == FINISHING) {
      S.state = CANCELLING;
    } else if (S.state == DONE) {
      S.state = FREE;
      srv->free_slots.push_back(it->second);
    }
    srv->ticket_slot.erase(it);
    srv->cancelled++;
    return RTS_OK;
  });
}

rts_status rts_server_get_stats(rts_server *srv, rts_server_stats *st) {
  return srv_guarded(srv, [&]() -> rts_status {
    if (!srv || !st) return fail(srv, RTS_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    memset(st, 0, sizeof *st);
    st->submitted = srv->submitted;
    st->completed = srv->completed;
    st->rejected = srv->rejected;
    st->cancelled = srv->cancelled;
    st->steps = srv->steps;
    st->queued = srv->queue.size();
    int active = 0;
    for (auto &S : srv->slots) active += S.state == ACTIVE;
    st->active = (uint32_t)active;
    st->p50_ms = percentile(srv->latencies, 0.50) * 1e3;
    st->p99_ms = percentile(srv->latencies, 0.99) * 1e3;
    st->p999_ms = percentile(srv->latencies, 0.999) * 1e3;
    double mx = 0, sum = 0;
    for (double v : srv->latencies) {
      mx = std::max(mx, v);
      sum += v;
    }
    st->max_ms = mx * 1e3;
    st->mean_ms = srv->latencies.empty() ? 0 : sum / (double)srv->latencies.size() * 1e3;
    st->plans = srv->plans;
    st->plan_ms_total = srv->plan_s * 1e3;
    return RTS_OK;
  });
}

rts_status rts_server_stop(rts_server *srv) {
  if (!srv) return RTS_OK;
  bool had_fatal = false;
  std::string msg;
  try {
    std::lock_guard<std::mutex> lk(srv->mu);
    had_fatal = !srv->fatal.empty();
    if (had_fatal) msg = "server had stopped: " + srv->fatal;
  } catch (const std::exception &) {
  }
  delete srv;  // nothing below touches the server
  if (!had_fatal) return RTS_OK;
  try {
    return rts::set_thread_error(RTS_ERR_CUDA, msg);
  } catch (const std::exception &) {
    return RTS_ERR_CUDA;
  }
}

// Open-loop replay for benchmarks: request q is submitted at arrival_s[q]
// seconds after the call starts, and its result slot is released as soon
// as it is done.  latency_ms[q] receives submit-to-done time (or -1 when
// the queue was full).  Blocks until every request is done.  A replay that
// stops on an error (a request the server refuses, a failed release)
// cancels its requests still in flight before it returns.
rts_status rts_server_replay(rts_server *srv, const rts_term *terms, const int32_t *offsets, int32_t nq,
                             const double *arrival_s, double *latency_ms) {
  return srv_guarded(srv, [&]() -> rts_status {
    rts::Range nvtx_range_("rts_server_replay");
    if (!srv || nq < 0 || (nq > 0 && (!offsets || !arrival_s || !latency_ms)))
      return fail(srv, RTS_ERR_ARG, "bad replay arguments");
    std::unordered_map<uint64_t, int> index_of;  // ticket -> query, filled by the producer
    std::vector<double> t_sub(nq, 0);
    std::atomic<int> produced{0};
    std::atomic<int> rejected{0};
    std::atomic<rts_status> prod_err{RTS_OK};  // written by the producer, read by the consumer
    std::mutex map_mu;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->track_done = true;
      srv->done_tickets.clear();
    }
    const double t0 = now_s();
    std::thread producer([&] {
      try {
        for (int q = 0; q < nq; q++) {
          const double due = t0 + arrival_s[q];
          while (now_s() < due) {
            const double left = due - now_s();
            if (left > 2e-4) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)(left * 5e5)));
          }
          t_sub[q] = now_s();
          uint64_t tk = 0;
          std::lock_guard<std::mutex> ml(map_mu);  // the consumer may look the ticket up right away
          const rts_status rc = rts_server_submit(srv, terms + offsets[q], offsets[q + 1] - offsets[q], &tk);
          if (rc == RTS_ERR_FULL) {
            latency_ms[q] = -1;
            rejected++;
          } else if (rc != RTS_OK) {
            prod_err.store(rc);
            produced.store(nq);
            return;
          } else {
            index_of[tk] = q;
          }
          produced.store(q + 1);
        }
      } catch (const std::exception &) {  // no exception may leave the thread
        prod_err.store(RTS_ERR_NOMEM);
        produced.store(nq);
      }
    });
    // join the producer on every way out, before the state it uses goes away
    struct Joiner {
      std::thread &t;
      ~Joiner() {
        if (t.joinable()) t.join();
      }
    } join_producer{producer};
    // consumer: release every finished request as it completes
    int finished = 0;
    rts_status rc = RTS_OK;
    while (rc == RTS_OK) {
      std::vector<std::pair<uint64_t, double>> batch;
      {
        std::unique_lock<std::mutex> lk(srv->mu);
        if (srv->done_tickets.empty()) srv->cv_done.wait_for(lk, std::chrono::milliseconds(1));
        if (!srv->fatal.empty()) {
          rc = RTS_ERR_CUDA;
          break;
        }
        batch.swap(srv->done_tickets);
      }
      for (auto &d : batch) {
        int q;
        {
          std::lock_guard<std::mutex> ml(map_mu);
          auto it = index_of.find(d.first);
          if (it == index_of.end()) continue;  // not one of this replay's requests
          q = it->second;
        }
        rc = rts_server_fetch(srv, d.first, nullptr, nullptr);
        if (rc != RTS_OK) break;  // the ticket stays listed and is cancelled below
        {
          std::lock_guard<std::mutex> ml(map_mu);
          index_of.erase(d.first);
        }
        latency_ms[q] = (d.second - t_sub[q]) * 1e3;
        finished++;
      }
      if (prod_err.load() != RTS_OK) rc = prod_err.load();
      if (produced.load() == nq && finished + rejected.load() == nq) break;
    }
    producer.join();
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->track_done = false;
      srv->done_tickets.clear();
    }
    if (rc == RTS_OK) rc = prod_err.load();
    // stopped early: release this replay's requests still queued, running or
    // done, so that their result slots return to the pool
    if (rc != RTS_OK) {
      std::lock_guard<std::mutex> ml(map_mu);
      for (auto &kv : index_of) rts_server_cancel(srv, kv.first);
      index_of.clear();
    }
    if (rc != RTS_OK && rc != RTS_ERR_CUDA) return rc;
    if (rc == RTS_ERR_CUDA) return fail(srv, rc, "server stopped: " + srv->fatal);
    return RTS_OK;
  });
}

}  // extern "C"
