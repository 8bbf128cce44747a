// CPU check of the batch planner (compiled and run by
// tests/test_planner_cpu.py; no GPU needed).  It includes the planner's
// translation unit, builds plans for seeded random batches on a context
// that has column pointers but no device (planning reads the pointers and
// the launch configuration only), and checks every plan:
//   * every kernel query sits in exactly one pass, no other query in any;
//   * pass sizes: term-by-term passes of at most kFewMaxQueries queries,
//     table passes of more, in the smallest of the 128/256/512-slot shapes;
//   * term-by-term passes carry each query's terms (always-true elsewhere);
//   * table passes: boundaries sorted and distinct, bmin/bmax their ends,
//     every mask bit of every used slot equal to the query's verdict on the
//     interval, every bucket of the index bracketing the true position of
//     the values it maps, and the pass fitting shared memory;
//   * shared positions: every union position and map entry against each
//     pass's own search;
//   * dropping queries from a plan (a server's finished requests) leaves no
//     slot naming them and every other slot as it was;
//   * a host-buffer batch's packed row chunk (nonzero-word mask, then the
//     nonzero words) expands to the chunk's words and writes nothing past it.
// Usage: planner_check SEED TRIALS; exit status 0 when every check holds.
#include "../rtscan_b200/csrc/batch.cu"

#include <cstdio>
#include <random>

namespace {

int g_fails = 0;
uint64_t g_table_passes = 0, g_few_passes = 0, g_kernel_queries = 0, g_bits = 0;
#define CHECK(cond, ...)                     \
  do {                                       \
    if (!(cond)) {                           \
      std::fprintf(stderr, __VA_ARGS__);     \
      std::fprintf(stderr, "\n");            \
      if (++g_fails > 20) std::exit(1);      \
    }                                        \
  } while (0)

constexpr uintptr_t kColStride = 0x100000;
constexpr uint32_t kMax = 0xFFFFFFFFu;

int column_of(const uint32_t *p) { return (int)((uintptr_t)p / kColStride) - 1; }

// The normalized term of query q on table column col: (lo, hi), or the
// whole domain when q does not constrain it.
void term_on(const rts::NormQuery &q, int col, uint32_t *lo, uint32_t *hi) {
  *lo = 0;
  *hi = kMax;
  for (size_t k = 0; k < q.cols.size(); k++)
    if (q.cols[k] == col) {
      *lo = q.lo[k];
      *hi = q.hi[k];
    }
}

void check_table_pass(const rts::BatchPlan &plan, const rts::BatchPlan::Pass &b, const std::vector<rts::NormQuery> &norm,
                      std::vector<int> &seen, std::mt19937_64 &rng) {
  const rts::BatchPass &bp = b.bp;
  const uint32_t *blob = plan.blob.data() + b.off;
  g_table_passes++;
  const int G = b.groups;
  const int32_t *slot = reinterpret_cast<const int32_t *>(blob + bp.slot_off);
  int nq = 0;
  for (int s = 0; s < 32 * G; s++) nq += slot[s] >= 0;
  CHECK(G == 4 || G == 8 || G == 16, "table pass with %d groups", G);
  CHECK(nq > rts::kFewMaxQueries, "table pass of %d queries", nq);
  CHECK(rts::pass_groups(nq) == G, "%d queries in a %d-group pass", nq, G);
  CHECK(b.warps == 8 || b.warps == 16, "pass planned for %d warps", b.warps);
  CHECK(rts::pass_smem4(bp.blob_words, bp.ncols <= 4 ? 4 : 8, G, b.warps) <= 227 * 1024,
        "pass needs %zu bytes of shared memory", rts::pass_smem4(bp.blob_words, bp.ncols <= 4 ? 4 : 8, G, b.warps));
  for (int s = 0; s < 32 * G; s++)
    if (slot[s] >= 0) {
      CHECK(slot[s] < (int)seen.size(), "slot maps to query %d", slot[s]);
      if (slot[s] < (int)seen.size()) seen[slot[s]]++;
    }
  for (int c = 0; c < bp.ncols; c++) {
    const int col = column_of(bp.col[c]);
    const uint32_t m = bp.m[c];
    const uint32_t *B = blob + bp.bnd_off[c];
    const uint32_t *tab = blob + bp.tab_off[c];
    for (uint32_t i = 1; i < m; i++) CHECK(B[i - 1] < B[i], "boundaries not increasing at %u", i);
    if (m) {
      CHECK(bp.bmin[c] == B[0] && bp.bmax[c] == B[m - 1], "bmin/bmax");
      CHECK(B[0] >= 1, "boundary 0");
    }
    // mask bits: interval pos holds [B[pos-1], B[pos]); its first value stands for it
    for (uint32_t pos = 0; pos <= m; pos++) {
      const uint32_t v = pos == 0 ? 0u : B[pos - 1];
      for (int s = 0; s < 32 * G; s++) {
        if (slot[s] < 0) continue;
        uint32_t lo, hi;
        term_on(norm[slot[s]], col, &lo, &hi);
        const bool want = lo <= v && v <= hi;
        const bool got = (tab[(size_t)pos * G + (s >> 5)] >> (s & 31)) & 1u;
        g_bits++;
        CHECK(want == got, "column %d pos %u slot %d: bit %d, query [%u, %u] at %u", col, pos, s, got, lo, hi, v);
      }
    }
    // bucket index: the bucket of x brackets #{B <= x}
    if (m) {
      const uint16_t *bk = reinterpret_cast<const uint16_t *>(blob + bp.bkt_off[c]);
      std::vector<uint32_t> xs;
      for (uint32_t i = 0; i < m; i++) {
        xs.push_back(B[i]);
        if (B[i] > 0) xs.push_back(B[i] - 1);
        if (B[i] < kMax) xs.push_back(B[i] + 1);
      }
      std::uniform_int_distribution<uint64_t> any(bp.bmin[c], bp.bmax[c]);
      for (int r = 0; r < 64; r++) xs.push_back((uint32_t)any(rng));
      for (uint32_t x : xs) {
        if (x < bp.bmin[c] || x >= bp.bmax[c]) continue;
        const uint32_t v = x - bp.bmin[c];
        const uint32_t k = bp.lgm[c] ? rts::bucket_of(v, bp.lgm[c]) : v >> bp.shift[c];
        CHECK(k < bp.nbk[c], "column %d value %u in bucket %u of %u", col, x, k, bp.nbk[c]);
        if (k >= bp.nbk[c]) continue;
        const uint32_t P = (uint32_t)(std::upper_bound(B, B + m, x) - B);
        CHECK(bk[k] <= P && P <= bk[k + 1], "column %d value %u: position %u outside bucket %u [%u, %u]", col, x, P, k,
              bk[k], bk[k + 1]);
      }
    }
  }
}

uint64_t g_pre_plans = 0, g_pre_lookups = 0;

// Shared positions: for values around every union boundary and at random,
// the union position (checked against the union bucket index) mapped through
// each fed pass's table gives the table word offset the pass would find by
// its own search (tab_off + #{pass boundaries <= x} * groups).
// Values to look up in a union column: both domain ends, every boundary and
// its neighbours, and random values.
std::vector<uint32_t> probe_values(const uint32_t *B, uint32_t m, std::mt19937_64 &rng) {
  std::vector<uint32_t> xs = {0u, 1u, kMax - 1, kMax};
  for (uint32_t i = 0; i < m; i++) {
    xs.push_back(B[i]);
    if (B[i]) xs.push_back(B[i] - 1);
    if (B[i] < kMax) xs.push_back(B[i] + 1);
  }
  for (int r = 0; r < 64; r++) xs.push_back((uint32_t)rng() >> (rng() % 32));
  return xs;
}

// The bucket index of one union column: pre_position equals the number of
// boundaries <= x for every probe value.
void check_pre_column(const rts::PreCol &pc, const uint32_t *ub, std::mt19937_64 &rng) {
  const uint32_t *B = ub + pc.bnd_off;
  CHECK(pc.nbk >= 1 && pc.nbk <= rts::kPreMaxBuckets, "union column with %u buckets", pc.nbk);
  for (uint32_t i = 1; i < pc.m; i++) CHECK(B[i - 1] < B[i], "union boundaries not sorted and distinct");
  for (uint32_t x : probe_values(B, pc.m, rng)) {
    const uint32_t want = (uint32_t)(std::upper_bound(B, B + pc.m, x) - B);
    const uint32_t got = rts::pre_position(pc, ub, x);
    CHECK(got == want, "union column (M %u L %u origin %u, %u buckets, m %u) value %u: position %u, want %u", pc.M,
          pc.L, pc.origin, pc.nbk, pc.m, x, got, want);
    g_pre_lookups++;
  }
}

void check_pre(const rts::BatchPlan &plan, std::mt19937_64 &rng) {
  const rts::PreParams &P = plan.pre;
  if (P.npass == 0) {
    for (const auto &b : plan.passes) CHECK(b.pre_slot < 0, "a pass fed by shared positions the plan does not have");
    return;
  }
  g_pre_plans++;
  CHECK(P.npass >= 1 && P.npass <= rts::kMaxPrePasses, "%d passes share positions", P.npass);
  CHECK(P.ncols >= 1 && P.ncols <= 4, "%d union columns", P.ncols);
  const uint32_t *ub = plan.blob.data() + plan.pre_off;
  const int NW = (P.npass + 1) / 2;
  CHECK(P.blob_words * 4 <= 200 * 1024 && plan.pre_off + P.blob_words <= plan.blob.size(), "union blob of %u words",
        P.blob_words);
  for (int c = 0; c < P.ncols; c++) check_pre_column(P.c[c], ub, rng);
  int fed = 0;
  for (const auto &b : plan.passes) {
    if (b.pre_slot < 0) continue;
    fed++;
    const int q = b.pre_slot;
    CHECK(q < P.npass, "pass slot %d of %d", q, P.npass);
    CHECK(!b.few && b.variant == 4 && b.cmax == 4 && b.groups >= 4, "shared positions feed a pass of shape %d/%d",
          b.cmax, b.groups);
    CHECK(b.bp.ncols == P.ncols, "a pass of %d columns fed by %d union columns", b.bp.ncols, P.ncols);
    const uint32_t *pblob = plan.blob.data() + b.off;
    for (int c = 0; c < b.bp.ncols && c < P.ncols; c++) {
      const rts::PreCol &pc = P.c[c];
      CHECK(pc.col == b.bp.col[c], "pass column %d is not union column %d", c, c);
      const uint32_t *Bu = ub + pc.bnd_off;
      const uint32_t *Bp = pblob + b.bp.bnd_off[c];
      const uint32_t mp = b.bp.m[c];
      for (uint32_t x : probe_values(Bu, pc.m, rng)) {
        const uint32_t upos = (uint32_t)(std::upper_bound(Bu, Bu + pc.m, x) - Bu);
        const uint32_t ppos = (uint32_t)(std::upper_bound(Bp, Bp + mp, x) - Bp);
        const uint32_t want = b.bp.tab_off[c] + ppos * (uint32_t)b.groups;
        const uint32_t got = (ub[pc.map_off + upos * NW + q / 2] >> (16 * (q & 1))) & 0xFFFFu;
        CHECK(got == want, "pass %d column %d value %u: offset %u, want %u", q, c, x, got, want);
        g_pre_lookups++;
      }
    }
  }
  CHECK(fed == P.npass, "%d passes fed, %d planned", fed, P.npass);
}

// batch_plan_drop: a random part of the plan's queries dropped (each a
// second time too), after which no slot of any pass names a dropped query,
// every other slot keeps its query, and every reported word is -1 in the
// blob.
uint64_t g_dropped = 0;
void check_drop(rts::BatchPlan &plan, int nq, std::mt19937_64 &rng) {
  auto slots_of = [&](std::vector<int> &owner) {  // query of every slot, in pass order
    owner.clear();
    for (const auto &b : plan.passes) {
      if (b.few) {
        for (int j = 0; j < b.fp.nq; j++) owner.push_back(b.fp.slot_query[j]);
      } else {
        const int32_t *slot = reinterpret_cast<const int32_t *>(plan.blob.data() + b.off + b.bp.slot_off);
        for (int sl = 0; sl < 32 * b.groups; sl++) owner.push_back(slot[sl]);
      }
    }
  };
  std::vector<int> before, after;
  slots_of(before);
  std::vector<char> gone(nq, 0);
  std::vector<uint32_t> words;
  for (int q = 0; q < nq; q++)
    if (rng() % 3 == 0) {
      gone[q] = 1;
      rts::batch_plan_drop(plan, q, words);
      rts::batch_plan_drop(plan, q, words);  // a second drop changes nothing
      g_dropped++;
    }
  rts::batch_plan_drop(plan, nq + 5, words);  // a query the plan does not hold
  slots_of(after);
  CHECK(before.size() == after.size(), "slot count changed");
  for (size_t i = 0; i < before.size() && i < after.size(); i++) {
    const int q = before[i];
    const int want = q >= 0 && q < nq && gone[q] ? -1 : q;
    CHECK(after[i] == want, "slot %zu: query %d after drops, want %d", i, after[i], want);
  }
  std::sort(words.begin(), words.end());
  CHECK(std::adjacent_find(words.begin(), words.end()) == words.end(), "a blob word reported twice");
  for (uint32_t w : words) CHECK(w < plan.blob.size() && plan.blob[w] == 0xFFFFFFFFu, "word %u not cleared", w);
}

// Bucket indexes of crafted boundary sets: single boundaries at the domain
// ends, dense runs, wide spreads, and runs crowded into one octave.
void check_pre_buckets(std::mt19937_64 &rng) {
  std::vector<std::vector<uint32_t>> sets = {
      {0}, {1}, {kMax}, {0, kMax}, {0, 1, 2, 3}, {kMax - 3, kMax - 2, kMax - 1, kMax}, {1u << 31}};
  std::vector<uint32_t> dense, wide, octave, skew, big;
  for (uint32_t i = 0; i < 3000; i++) dense.push_back(1000 + i);
  for (uint32_t i = 0; i < 2000; i++) wide.push_back((uint32_t)rng());
  for (uint32_t i = 0; i < 1500; i++) octave.push_back((1u << 30) + (uint32_t)(rng() % (1u << 20)));
  for (uint32_t i = 0; i < 2500; i++) skew.push_back((uint32_t)rng() >> (rng() % 32));
  for (uint32_t i = 0; i < 65535; i++) big.push_back(i * 65537u);
  for (auto *v : {&dense, &wide, &octave, &skew, &big}) sets.push_back(*v);
  for (auto &B : sets) {
    std::sort(B.begin(), B.end());
    B.erase(std::unique(B.begin(), B.end()), B.end());
    rts::PreCol pc;
    std::memset(&pc, 0, sizeof pc);
    std::vector<uint32_t> ub = rts::pre_buckets(B, pc);
    pc.bkt_off = 0;
    pc.bnd_off = (uint32_t)ub.size();
    ub.insert(ub.end(), B.begin(), B.end());
    check_pre_column(pc, ub.data(), rng);
  }
}

uint64_t g_expanded = 0;
// Chunks of random length and density, packed as pack_kernel lays them out
// (bit k of mask word i set when word 32i + k is nonzero; the nonzero words
// follow in order), expanded by the host's expand_mask into a buffer of ones.
void check_expand_mask(std::mt19937_64 &rng) {
  const uint64_t lens[] = {1, 31, 32, 33, 1000, 4096, 4097, 65536 + 17};
  for (uint64_t cw : lens)
    for (int density : {0, 1, 8, 64, 200, 256}) {  // nonzero words per 256
      std::vector<uint32_t> words(cw);
      for (auto &w : words) w = (int)(rng() % 256) < density ? (uint32_t)(rng() | 1) : 0u;
      if (density == 256 && cw > 40) words[cw / 2] = 0;  // one zero among full mask words
      const uint64_t nm = (cw + 31) / 32;
      std::vector<uint32_t> packed(nm, 0u);
      for (uint64_t i = 0; i < cw; i++)
        if (words[i]) {
          packed[i / 32] |= 1u << (i % 32);
          packed.push_back(words[i]);
        }
      for (int off = 0; off < 4; off++) {  // destinations at every 4-byte offset from a 16-byte boundary
        std::vector<uint32_t> out(cw + 16, 0xFFFFFFFFu);
        uint32_t *base = out.data();
        while ((uintptr_t)base & 15) base++;
        rts::expand_mask(base + off, cw, packed.data());
        CHECK(std::equal(words.begin(), words.end(), base + off), "expand_mask: %llu words, density %d, offset %d differ",
              (unsigned long long)cw, density, off);
        for (uint32_t *w = out.data(); w < out.data() + out.size(); w++)
          CHECK(*w == 0xFFFFFFFFu || (w >= base + off && w < base + off + cw),
                "expand_mask: %llu words, density %d, offset %d: a word outside the chunk written",
                (unsigned long long)cw, density, off);
        g_expanded += cw;
      }
    }
}

void check_few_pass(const rts::BatchPlan::Pass &b, const std::vector<rts::NormQuery> &norm, std::vector<int> &seen) {
  const rts::FewPass &f = b.fp;
  g_few_passes++;
  CHECK(f.nq >= 1 && f.nq <= rts::kFewMaxQueries, "term-by-term pass of %d queries", f.nq);
  for (int j = 0; j < f.nq; j++) {
    const int q = f.slot_query[j];
    CHECK(q >= 0 && q < (int)seen.size(), "few slot maps to query %d", q);
    if (q < 0 || q >= (int)seen.size()) continue;
    seen[q]++;
    for (int c = 0; c < f.ncols; c++) {
      uint32_t lo, hi;
      term_on(norm[q], column_of(f.col[c]), &lo, &hi);
      CHECK(f.term[j][c].x == lo && f.term[j][c].y == hi - lo, "few pass: query %d column %d term", q, c);
    }
  }
}

uint32_t draw_bound(std::mt19937_64 &rng, const std::vector<uint32_t> &pool) {
  std::uniform_int_distribution<int> pick(0, 3);
  if (pick(rng) == 0) return (uint32_t)rng();
  return pool[std::uniform_int_distribution<size_t>(0, pool.size() - 1)(rng)];
}

}  // namespace

int main(int argc, char **argv) {
  const uint64_t seed = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1;
  const int trials = argc > 2 ? std::atoi(argv[2]) : 20;
  std::mt19937_64 rng(seed);
  check_pre_buckets(rng);
  std::mt19937_64 pack_rng(seed ^ 0x5eed5eedull);  // the trials' own stream is left as it was
  check_expand_mask(pack_rng);
  const int counts[] = {1, 2, 3, 4, 20, 21, 32, 100, 128, 129, 200, 256, 257, 400, 512, 513, 700, 1100};
  for (int t = 0; t < trials; t++) {
    auto *ctx = new rts_ctx();  // never destroyed: it owns no device memory
    // every fifth trial: at most four columns and several passes' worth of
    // queries, the plans whose passes share positions
    const bool shared = t % 5 == 4;
    const int ncols = shared ? 1 + (int)(rng() % 4) : 1 + (int)(rng() % 10);
    for (int c = 0; c < ncols; c++) ctx->cols.push_back(reinterpret_cast<const uint32_t *>(kColStride * (c + 1)));
    ctx->nrows = 1 << 20;
    ctx->sm_count = 148;
    const size_t budgets[] = {136 * 1024, 64 * 1024, 8 * 1024};
    ctx->batch_cfg.table_budget = budgets[rng() % 3];
    ctx->batch_cfg.warps_per_cta = rng() % 2 ? 16 : 8;  // 8-warp passes fit more blob beside a smaller stage
    const int nq = shared   ? 600 + (int)(rng() % 500)
                   : rng() % 4 ? counts[rng() % (sizeof counts / sizeof counts[0])]
                               : 1 + (int)(rng() % 1100);
    // bounds from a small pool (shared boundaries, domain edges) and random values
    std::vector<uint32_t> pool = {0, 1, 2, kMax - 1, kMax, 1u << 31};
    // (every tenth trial a pool of 1500, so that the union columns hold
    // hundreds of boundaries, crowded buckets among them)
    const int npool = shared && t % 10 == 9 ? 1500 : 40;
    for (int i = 0; i < npool; i++) pool.push_back((uint32_t)rng() >> (rng() % 32));
    std::vector<rts_term> terms;
    std::vector<int32_t> offsets = {0};
    for (int q = 0; q < nq; q++) {
      const int k = 1 + (int)(rng() % std::min(ncols, 9));
      for (int i = 0; i < k; i++) {
        rts_term tm;
        tm.column = (int32_t)(rng() % ncols);
        uint32_t a = draw_bound(rng, pool), b = draw_bound(rng, pool);
        if (rng() % 8 && a > b) std::swap(a, b);  // now and then an empty term
        tm.lo = a;
        tm.hi = b;
        terms.push_back(tm);
      }
      offsets.push_back((int32_t)terms.size());
    }
    std::vector<rts::NormQuery> norm = rts::normalize_all(ctx, terms.data(), offsets.data(), nq);
    std::vector<int> inside;
    for (int q = 0; q < nq; q++)
      if (rts::runs_in_kernel(norm[q])) inside.push_back(q);
    g_kernel_queries += inside.size();
    std::vector<int> seen(nq, 0);
    if (!inside.empty()) {
      rts::BatchPlanPtr plan = rts::make_batch_plan(ctx, norm, inside, nullptr, ctx->batch_cfg.table_budget, true);
      for (const auto &b : plan->passes) {
        if (b.few) check_few_pass(b, norm, seen);
        else check_table_pass(*plan, b, norm, seen, rng);
      }
      check_pre(*plan, rng);
      std::mt19937_64 drop_rng(seed * 1000003ull + (uint64_t)t);  // the trials' own stream is left as it was
      check_drop(*plan, nq, drop_rng);
    }
    for (int q = 0; q < nq; q++) {
      const int want = rts::runs_in_kernel(norm[q]) ? 1 : 0;
      CHECK(seen[q] == want, "trial %d: query %d in %d passes (want %d)", t, q, seen[q], want);
    }
  }
  if (g_fails) {
    std::fprintf(stderr, "%d checks failed\n", g_fails);
    return 1;
  }
  std::printf("planner ok: %d trials, seed %llu: %llu kernel queries, %llu table passes, %llu term-by-term passes, "
              "%llu mask bits, %llu plans with shared positions (%llu lookups), %llu queries dropped, "
              "%llu packed words expanded\n",
              trials, (unsigned long long)seed, (unsigned long long)g_kernel_queries, (unsigned long long)g_table_passes,
              (unsigned long long)g_few_passes, (unsigned long long)g_bits, (unsigned long long)g_pre_plans,
              (unsigned long long)g_pre_lookups, (unsigned long long)g_dropped,
              (unsigned long long)g_expanded);
  return 0;
}
