// CPU check of the BinDex query planner's host steps (compiled and run by
// tests/test_planner_cpu.py; no GPU needed).  It includes the BinDex
// translation unit and, for seeded random sorted columns (duplicates,
// narrow and wide domains) and random bounds, checks:
//   * estimate(): the search window [wlo, whi] it returns from the sample of
//     every 1024th sorted value contains lower_bound(sorted, b), and its
//     estimate lies in the window;
//   * nearest(): the filter vector (or constant) it picks has the smallest
//     rank distance to the estimate among the constant zero (rank 0), the
//     constant one (rank n) and every filter vector k (rank first_rank[k+1]).
// Usage: bindex_plan_check SEED TRIALS; exit status 0 when every check holds.
#include "../rtscan_b200/csrc/bindex.cu"

#include <cstdio>
#include <random>

int main(int argc, char **argv) {
  const uint64_t seed = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1;
  const int trials = argc > 2 ? std::atoi(argv[2]) : 20;
  std::mt19937_64 rng(seed);
  int fails = 0;
  uint64_t bounds = 0;
  for (int t = 0; t < trials; t++) {
    auto *B = new rts::GpuBinDex();  // host fields only; never destroyed (no device memory)
    const uint64_t n = 1 + rng() % 300000;
    B->n = n;
    B->K = 2 + (int)(rng() % 255);
    const uint32_t domain = rng() % 3 == 0 ? 1 + (uint32_t)(rng() % 300) : 0xFFFFFFFFu;
    std::vector<uint32_t> S(n);
    for (auto &v : S) v = (uint32_t)(rng() % ((uint64_t)domain + 1));
    std::sort(S.begin(), S.end());
    for (uint64_t j = 0; j * rts::kSampleStride < n; j++) B->sample.push_back(S[j * rts::kSampleStride]);
    // area ranks as the build keeps them: lower_bound of each area's start value
    B->first_rank.resize(B->K);
    for (int k = 0; k < B->K; k++) {
      const uint32_t start = S[(uint64_t)k * (n / B->K) < n ? (uint64_t)k * (n / B->K) : n - 1];
      B->first_rank[k] = (uint64_t)(std::lower_bound(S.begin(), S.end(), start) - S.begin());
    }
    B->first_rank[0] = 0;
    for (int r = 0; r < 200; r++) {
      uint32_t b;
      switch (rng() % 4) {
        case 0: b = S[rng() % n]; break;
        case 1: b = S[rng() % n] + 1; break;
        case 2: b = S[rng() % n] - 1; break;
        default: b = (uint32_t)rng(); break;
      }
      const uint64_t L = (uint64_t)(std::lower_bound(S.begin(), S.end(), b) - S.begin());
      const rts::Est e = rts::estimate(*B, b);
      bounds++;
      if (!(e.wlo <= L && L <= e.whi && e.wlo <= e.est && e.est <= e.whi)) {
        std::fprintf(stderr, "trial %d: bound %u rank %llu outside window [%llu, %llu] (est %llu)\n", t, b,
                     (unsigned long long)L, (unsigned long long)e.wlo, (unsigned long long)e.whi,
                     (unsigned long long)e.est);
        if (++fails > 20) return 1;
      }
      const rts::Approx a = rts::nearest(*B, e.est);
      auto dist = [&](uint64_t r) { return r > e.est ? r - e.est : e.est - r; };
      uint64_t best = std::min(dist(0), dist(n));
      for (int k = 1; k < B->K; k++) best = std::min(best, dist(B->first_rank[k]));
      const uint64_t want_rank = a.k < 0 ? 0 : a.k >= B->K - 1 ? n : B->first_rank[a.k + 1];
      if (dist(a.rank) != best || a.rank != want_rank) {
        std::fprintf(stderr, "trial %d: nearest(%llu) picked k=%d rank %llu, best distance %llu\n", t,
                     (unsigned long long)e.est, a.k, (unsigned long long)a.rank, (unsigned long long)best);
        if (++fails > 20) return 1;
      }
    }
  }
  if (fails) {
    std::fprintf(stderr, "%d checks failed\n", fails);
    return 1;
  }
  std::printf("bindex planner ok: %d trials, seed %llu: %llu bounds\n", trials, (unsigned long long)seed,
              (unsigned long long)bounds);
  return 0;
}
