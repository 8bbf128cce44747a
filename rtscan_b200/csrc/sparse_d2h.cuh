// Sparse result bitmaps leave the device as (word, value) pairs (included
// by batch.cu inside its anonymous namespace in rts; used by
// rts_scan_batch_host).
//
// A host-buffer batch call moves every query's bitmap over PCIe, which sets
// its time (12.5 MB per query at 1e8 rows; the scan itself is about 3 % of
// the call).  A bitmap of a selective query is mostly zero words: below
// about 0.9 % of the rows, at most one word in four is nonzero.  Per row
// chunk, after the chunk's scan:
//   * nnz_kernel counts each query's nonzero words in the chunk, and the
//     host reads the counts (4 bytes per query) while the next chunk runs;
//   * a query with at most one nonzero word in kSparseDensity (four) is
//     sent as the chunk's (word index, value) pairs in word order, packed by
//     pack_kernel at offsets the host assigns (8 bytes per nonzero word
//     instead of 4 per word), and expanded on the host by worker threads
//     (zeros between the pairs);
//   * every other query keeps its 2D copy, one per run of consecutive
//     dense queries.
// The host's memory takes the worker threads' writes beside the DMA
// (measured on the B200 box: 55 GB/s of memset beside a 45 GB/s
// device-to-host copy, against 52 GB/s for the copy alone).  On the bench
// workload (1e8 rows x 4 columns, 1024 queries) a call took 228 / 221 /
// 208-210 / 208 ms with a word in 16 / 8 / 4 / 3 nonzero as the limit.
#pragma once
// (<condition_variable>, <functional>, <mutex> and <thread> come from batch.cu.)

constexpr int kSparseThreads = 256;
constexpr int kSparseWordsPerThread = 4;
constexpr uint64_t kSparseMinWords = 4096;  // chunks of fewer words per query are sent whole
constexpr uint64_t kSparseDensity = 4;      // a packed chunk has at most one nonzero word in this many
constexpr uint64_t kSparseMaxPairs = 1ull << 24;  // pairs of one chunk (128 MiB per staging slot)

// Nonzero words of query q's bitmap in [w0, w1): one block per query.
__global__ void __launch_bounds__(kSparseThreads) nnz_kernel(const uint32_t *bm, uint64_t stride, uint64_t w0,
                                                             uint64_t w1, uint32_t *nnz) {
  const uint32_t *p = bm + (uint64_t)blockIdx.x * stride;
  uint32_t c = 0;
  for (uint64_t w = w0 + threadIdx.x; w < w1; w += 4 * kSparseThreads) {
    uint32_t v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint64_t wk = w + (uint64_t)k * kSparseThreads;
      v[k] = wk < w1 ? __ldg(p + wk) : 0u;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) c += v[k] != 0;
  }
  __shared__ uint32_t part[kSparseThreads / 32];
  c = __reduce_add_sync(0xFFFFFFFFu, c);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int i = 0; i < kSparseThreads / 32; i++) s += part[i];
    nnz[blockIdx.x] = s;
  }
}

// The nonzero words of query ql[j] in [w0, w1) as (word - w0, value) pairs
// in word order at out + off[j]: one block per listed query, tiles of
// kSparseThreads * kSparseWordsPerThread words, each thread four
// consecutive words, ranks by a block-wide prefix of the threads' counts.
__global__ void __launch_bounds__(kSparseThreads) pack_kernel(const uint32_t *bm, uint64_t stride, uint64_t w0,
                                                              uint64_t w1, const int32_t *ql, const uint64_t *off,
                                                              uint2 *out) {
  const uint32_t *p = bm + (uint64_t)ql[blockIdx.x] * stride;
  uint2 *o = out + off[blockIdx.x];
  __shared__ uint32_t wsum[kSparseThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t base = 0;
  constexpr uint64_t kTile = (uint64_t)kSparseThreads * kSparseWordsPerThread;
  for (uint64_t t0 = w0; t0 < w1; t0 += kTile) {
    const uint64_t w = t0 + (uint64_t)threadIdx.x * kSparseWordsPerThread;
    uint32_t v[kSparseWordsPerThread];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kSparseWordsPerThread; k++) {
      v[k] = w + k < w1 ? __ldg(p + w + k) : 0u;
      c += v[k] != 0;
    }
    uint32_t incl = c;  // inclusive prefix over the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= d) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int i = 0; i < kSparseThreads / 32; i++) {
      before += i < warp ? wsum[i] : 0u;
      total += wsum[i];
    }
    uint64_t r = base + before + incl - c;
#pragma unroll
    for (int k = 0; k < kSparseWordsPerThread; k++)
      if (v[k]) o[r++] = make_uint2((uint32_t)(w + k - w0), v[k]);
    base += total;
    __syncthreads();  // wsum is rewritten by the next tile
  }
}

// Host threads running queued tasks; the destructor runs what is queued and
// joins (so no task outlives the call that queued it).
class TaskPool {
 public:
  explicit TaskPool(int n) {
    for (int i = 0; i < n; i++) th_.emplace_back([this] { run(); });
  }
  ~TaskPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  void post(std::function<void()> f) {
    {
      std::lock_guard<std::mutex> g(mu_);
      q_.push_back(std::move(f));
    }
    cv_.notify_one();
  }
  int size() const { return (int)th_.size(); }

 private:
  void run() {
    for (;;) {
      std::function<void()> f;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [this] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;
        f = std::move(q_.front());
        q_.erase(q_.begin());
      }
      f();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<std::function<void()>> q_;
  std::vector<std::thread> th_;
  bool stop_ = false;
};

// Counter of unfinished tasks per host staging slot.
class SlotGate {
 public:
  void add(int slot, int n) {
    std::lock_guard<std::mutex> g(mu_);
    busy_[slot] += n;
  }
  void done(int slot) {
    {
      std::lock_guard<std::mutex> g(mu_);
      busy_[slot]--;
    }
    cv_.notify_all();
  }
  void wait_free(int slot) {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [&] { return busy_[slot] == 0; });
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  int busy_[8] = {0};
};

// Query q's chunk [w0, w0 + cw) of the host bitmap from its pairs: zeros
// between them.
inline void expand_pairs(uint32_t *dst, uint64_t cw, const uint2 *pairs, uint64_t n) {
  uint64_t cur = 0;
  for (uint64_t i = 0; i < n; i++) {
    const uint64_t w = pairs[i].x;
    if (w > cur) memset(dst + cur, 0, (w - cur) * 4);
    dst[w] = pairs[i].y;
    cur = w + 1;
  }
  if (cur < cw) memset(dst + cur, 0, (cw - cur) * 4);
}
