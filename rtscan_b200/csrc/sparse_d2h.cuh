// Sparse result bitmaps leave the device packed as a nonzero-word mask and
// the nonzero words (included by batch.cu inside its anonymous namespace in
// rts; used by rts_scan_batch_host).
//
// A host-buffer batch call moves every query's bitmap over PCIe, which sets
// its time (12.5 MB per query at 1e8 rows; the scan itself is about 3 % of
// the call).  A bitmap of a selective query is mostly zero words.  Per row
// chunk, after the chunk's scan:
//   * nnz_kernel counts each query's nonzero words in the chunk, and the
//     host reads the counts (4 bytes per query) while the next chunk runs;
//   * a query whose mask (one bit per word) and nonzero words take at most
//     kPackNum / kPackDen (3/8) of the chunk's words is packed by
//     pack_kernel at the offset the host assigns, and expanded on the host
//     by worker threads (zeros where the mask bit is clear);
//   * every other query keeps its 2D copy, one per run of consecutive
//     dense queries.
// The host's memory takes the worker threads' writes beside the DMA
// (measured on the B200 box: 55 GB/s of memset beside a 45 GB/s
// device-to-host copy, against 52 GB/s for the copy alone).
#pragma once
// (<condition_variable>, <functional>, <mutex> and <thread> come from batch.cu.)

constexpr int kSparseThreads = 256;
constexpr int kSparseWordsPerThread = 4;
constexpr uint64_t kSparseMinWords = 4096;  // chunks of fewer words per query are sent whole
// a chunk is packed when its mask and values take at most kPackNum /
// kPackDen of its words
constexpr uint64_t kPackNum = 3, kPackDen = 8;
constexpr uint64_t kSparseMaxWords = 1ull << 25;  // packed words of one chunk (128 MiB per staging slot)

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

// Query ql[j]'s words [w0, w1) as a nonzero mask (bit k of mask word i:
// word 32i + k is nonzero) followed by the nonzero words in order, at
// out + off[j]: one block per listed query, one word per thread per tile of
// kPackThreads words, a warp's ballot its mask word, ranks by a block-wide
// prefix of the warps' counts.
constexpr int kPackThreads = 1024;
__global__ void __launch_bounds__(kPackThreads) pack_kernel(const uint32_t *bm, uint64_t stride, uint64_t w0,
                                                            uint64_t w1, const int32_t *ql, const uint64_t *off,
                                                            uint32_t *out) {
  const uint32_t *p = bm + (uint64_t)ql[blockIdx.x] * stride + w0;
  const uint64_t cw = w1 - w0, nm = (cw + 31) / 32;
  uint32_t *mask = out + off[blockIdx.x];
  uint32_t *vals = mask + nm;
  __shared__ uint32_t wcnt[kPackThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t base = 0;
  for (uint64_t t0 = 0; t0 < cw; t0 += kPackThreads) {
    const uint64_t i = t0 + threadIdx.x;
    const uint32_t v = i < cw ? __ldg(p + i) : 0u;
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, v != 0);
    if (lane == 0) {
      if (t0 / 32 + warp < nm) mask[t0 / 32 + warp] = b;
      wcnt[warp] = __popc(b);
    }
    __syncthreads();
    uint32_t incl = wcnt[lane];  // every warp scans the warps' counts
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= d) incl += y;
    }
    const uint32_t before = __shfl_sync(0xFFFFFFFFu, incl, warp) - wcnt[warp];
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (v) vals[base + before + __popc(b & ((1u << lane) - 1u))] = v;
    base += total;
    __syncthreads();  // wcnt is rewritten by the next tile
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

// Query q's chunk of cw words of the host bitmap from its mask and values
// (pack_kernel's layout): the chunk is zeroed, then each set mask bit's word
// is stored.
inline void expand_mask(uint32_t *dst, uint64_t cw, const uint32_t *packed) {
  const uint64_t nm = (cw + 31) / 32;
  const uint32_t *vals = packed + nm;
  memset(dst, 0, cw * 4);
  for (uint64_t i = 0; i < nm; i++) {
    uint32_t *d = dst + 32 * i;
    for (uint32_t m = packed[i]; m; m &= m - 1) d[__builtin_ctz(m)] = *vals++;
  }
}
