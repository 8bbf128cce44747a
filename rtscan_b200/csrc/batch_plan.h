// Host-side planning interface of the batched kernel (batch.cu), shared
// with the serving loop (serve.cpp).
#pragma once

#include <memory>
#include <vector>

#include "rts_internal.h"

namespace rts {

// Vector with room for N elements in place, so that the usual query of a
// few terms is planned without heap allocations; it moves to the heap when
// it grows past N.
template <class T, int N>
class SmallVec {
 public:
  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T *data() { return big_ ? heap_.data() : inl_; }
  const T *data() const { return big_ ? heap_.data() : inl_; }
  T *begin() { return data(); }
  T *end() { return data() + n_; }
  const T *begin() const { return data(); }
  const T *end() const { return data() + n_; }
  T &operator[](size_t i) { return data()[i]; }
  const T &operator[](size_t i) const { return data()[i]; }
  void push_back(const T &x) {
    if (!big_ && n_ == (size_t)N) {
      heap_.assign(inl_, inl_ + N);
      big_ = true;
    }
    if (big_) heap_.push_back(x);
    else inl_[n_] = x;
    n_++;
  }

 private:
  T inl_[N];
  std::vector<T> heap_;
  size_t n_ = 0;
  bool big_ = false;
};

// A query after validation: terms merged per column (ranges intersected),
// always-true terms dropped.
struct NormQuery {
  int index = 0;                   // position in the caller's list
  SmallVec<int, 8> cols;           // constrained columns
  SmallVec<uint32_t, 8> lo, hi;
  bool empty = false;              // some term can never match
};

NormQuery normalize(const rts_term *terms, int n, int index, int ncols_table);
std::vector<NormQuery> normalize_all(rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int nq);
// True when the batched kernel answers the query (non-empty, 1..8 columns);
// the others go through launch_outside.
bool runs_in_kernel(const NormQuery &q);

// Answer queries `which` (indices into norm) over the whole table with fill
// or fused-scan launches; query qi writes bitmap / count out_index[qi] (qi
// when out_index is null).  Returns the kernels launched.
int launch_outside(rts_ctx *ctx, const std::vector<NormQuery> &norm, const std::vector<int> &which,
                   const int32_t *out_index, uint32_t *out, uint64_t stride_words, unsigned long long *counts,
                   cudaStream_t s);

// Mask-table passes for the kernel queries `which`, built on the host.
struct BatchPlan;
struct BatchPlanDeleter {
  void operator()(BatchPlan *p) const;
};
using BatchPlanPtr = std::unique_ptr<BatchPlan, BatchPlanDeleter>;
// share_positions: a plan of several table passes over four columns or
// fewer searches each row's positions once for all of them (a faster step
// for a little more host planning).
BatchPlanPtr make_batch_plan(rts_ctx *ctx, const std::vector<NormQuery> &norm, const std::vector<int> &which,
                             const int32_t *out_index, size_t table_budget, bool share_positions);
// The words to upload to the device before launching.
const std::vector<uint32_t> &batch_plan_blob(const BatchPlan &plan);
// Launch every pass over rows [row_begin, row_end) (row_begin a multiple of
// 4096) with the plan blob at dev_blob; counts are accumulated (not reset).
// scratch (scratch_bytes, the caller's, not used by another launch at the
// same time) holds the rows' shared positions when the plan has them and it
// is large enough (batch_plan_scratch_bytes); else every pass searches.
int launch_batch_plan(rts_ctx *ctx, BatchPlan &plan, const uint32_t *dev_blob, uint32_t *out,
                      uint64_t stride_words, unsigned long long *counts, uint64_t row_begin, uint64_t row_end,
                      void *scratch, size_t scratch_bytes, cudaStream_t s);
// Stop the plan from writing query qi's bitmap and count (a request that
// finished or was cancelled while the plan keeps running): term-by-term and
// fused passes are changed in the plan; for table passes the plan blob's
// slot entry becomes -1 and its word offset is appended to `blob_words`,
// the words the caller must also set to 0xFFFFFFFF in the uploaded blob
// before the next launch.  A query the plan does not hold is ignored.
void batch_plan_drop(BatchPlan &plan, int qi, std::vector<uint32_t> &blob_words);
// Scratch bytes that launch_batch_plan needs for `rows` rows (0: none); at
// most kMaxSharedPasses * (rows + 1) * 8 for any plan.
size_t batch_plan_scratch_bytes(const BatchPlan &plan, uint64_t rows);
constexpr int kMaxSharedPasses = 4;

}  // namespace rts
