// ref_harness.cpp -- THE ORACLE's link to the real reference.  Test
// infrastructure only; never part of the product.
//
// Drives the reference's own CPU path: bindex.cpp compiled unmodified from
// the reference source tree (its main() renamed by the recipe in
// oracle/Makefile) and linked with this driver.  The driver repeats the
// query loop of exp_opt (bindex.cpp:2157-2297) with the reference's own
// functions:
//   * stringSplit / get_target_numbers  (bindex.cpp:238-245, 1840-1849)
//   * init_bindex                       (bindex.cpp:599-671)
//   * bindex_scan_{lt,le,gt,ge,eq,bt}   (bindex.cpp:1365-1691)
//   * refine_result_bitmap (AND merge)  (bindex.cpp:1259-1281, driven as at 2240-2260)
//   * raw_scan_entry (scalar checker)   (bindex.cpp:1894-1957)
// and writes, per query, the BinDex bitmap, the scalar-filter bitmap and
// their counts, so the golden fixtures and the CPU baseline come from the
// reference itself.  Row count is compile-time (DATA_N), as in the reference.
//
// usage: ref_bindex_<N> -f <column file> -b <ncols> -p <scan_cmd>
//                       [-o <out dir>] [-r <repeats>] [-n <max queries>]
//                       [-c <checked queries>]
// -c k runs the scalar-filter check on the first k queries only (default:
// every query); a query left unchecked reports raw_hits -1 and equal -1.
// stdout, one line per query:
//   query <i> bindex_hits <a> raw_hits <b> equal <0|1|-1> scan_ms <t>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <chrono>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

typedef uint32_t CODE;
typedef unsigned int BITS;
typedef int POSTYPE;
struct BinDex;  // the reference's `typedef struct {...} BinDex;` (linkage name BinDex)
enum OPERATOR { EQ = 0, LT, GT, LE, GE, BT };

void init_bindex(BinDex *bindex, CODE *data, POSTYPE n);
void bindex_scan_lt(BinDex *, BITS *, CODE);
void bindex_scan_le(BinDex *, BITS *, CODE);
void bindex_scan_gt(BinDex *, BITS *, CODE);
void bindex_scan_ge(BinDex *, BITS *, CODE);
void bindex_scan_bt(BinDex *, BITS *, CODE, CODE);
void bindex_scan_eq(BinDex *, BITS *, CODE);
void refine_result_bitmap(BITS *bitmap_a, BITS *bitmap_b, int start_idx, int end_idx, int t_id);
void raw_scan_entry(std::vector<CODE> *target_l, std::vector<CODE> *target_r, std::string search_cmd,
                    BinDex *bindex, BITS *bitmap, BITS *mergeBitmap, CODE *raw_data);
std::vector<std::string> stringSplit(const std::string &str, char delim);
std::vector<CODE> get_target_numbers(std::string s);

#ifndef DATA_N
#error "DATA_N must be given, as for the reference"
#endif
static const int kN = (int)DATA_N;
static const int kThreads = 20;  // THREAD_NUM, bindex.cpp:27
static const size_t kBinDexBytes = 1 << 20;  // >= sizeof(BinDex) for any VAREA_N <= 8192

static int words_for(int n) { return (n + 31) / 32; }

static uint64_t count_bits(const BITS *bm, int n) {
  uint64_t c = 0;
  for (int i = 0; i < n; i++) c += (bm[i >> 5] >> (31 - (i & 31))) & 1u;
  return c;
}

// The AND merge of exp_opt, bindex.cpp:2237-2260: 20 strided threads.
static void and_merge(BITS *dst, BITS *src) {
  int max_idx = words_for(kN);
  int stride = (max_idx + kThreads - 1) / kThreads;
  std::vector<std::thread> th;
  int start = 0, end = 0, t = 0;
  while (end < max_idx && t < kThreads) {
    end = start + stride;
    if (end > max_idx) end = max_idx;
    th.emplace_back(refine_result_bitmap, dst, src, start, end, t);
    start += stride;
    t++;
  }
  for (auto &x : th) x.join();
}

static void run_op(BinDex *b, BITS *bm, const std::string &cmd, CODE t1, CODE t2) {
  if (cmd == "lt") bindex_scan_lt(b, bm, t1);
  else if (cmd == "le") bindex_scan_le(b, bm, t1);
  else if (cmd == "gt") bindex_scan_gt(b, bm, t1);
  else if (cmd == "ge") bindex_scan_ge(b, bm, t1);
  else if (cmd == "eq") bindex_scan_eq(b, bm, t1);
  else if (cmd == "bt") bindex_scan_bt(b, bm, t1, t2);
}

int main(int argc, char **argv) {
  char path[4096] = "", cmd_path[4096] = "", out_dir[4096] = "";
  int ncols = 1, repeats = 1, max_queries = 1 << 30, checked = 1 << 30;
  int opt;
  while ((opt = getopt(argc, argv, "f:b:p:o:r:n:c:")) != -1) {
    switch (opt) {
      case 'f': snprintf(path, sizeof path, "%s", optarg); break;
      case 'b': ncols = atoi(optarg); break;
      case 'p': snprintf(cmd_path, sizeof cmd_path, "%s", optarg); break;
      case 'o': snprintf(out_dir, sizeof out_dir, "%s", optarg); break;
      case 'r': repeats = atoi(optarg); break;
      case 'n': max_queries = atoi(optarg); break;
      case 'c': checked = atoi(optarg); break;
      default: fprintf(stderr, "unknown option\n"); return 2;
    }
  }
  if (!path[0] || !cmd_path[0] || ncols < 1 || repeats < 1) {
    fprintf(stderr, "usage: %s -f data -b ncols -p scan_cmd [-o dir] [-r repeats] [-n max_queries] [-c checked]\n",
            argv[0]);
    return 2;
  }
  FILE *fp = fopen(path, "rb");
  if (!fp) { fprintf(stderr, "cannot open %s\n", path); return 2; }
  std::vector<CODE *> data(ncols);
  for (int c = 0; c < ncols; c++) {
    data[c] = (CODE *)malloc((size_t)kN * sizeof(CODE));
    if (fread(data[c], sizeof(CODE), kN, fp) != (size_t)kN) { fprintf(stderr, "short read\n"); return 2; }
  }
  fclose(fp);

  std::vector<BinDex *> bindexs(ncols);
  auto t0 = std::chrono::steady_clock::now();
  for (int c = 0; c < ncols; c++) {
    bindexs[c] = (BinDex *)calloc(1, kBinDexBytes);
    init_bindex(bindexs[c], data[c], kN);
  }
  double build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  printf("build_ms %.3f\n", build_ms);

  int W = words_for(kN);
  size_t bytes = (((size_t)W * sizeof(BITS)) + 31) / 32 * 32;
  std::vector<BITS *> bm(ncols), chk(ncols);
  for (int c = 0; c < ncols; c++) {
    bm[c] = (BITS *)aligned_alloc(32, bytes);
    chk[c] = (BITS *)aligned_alloc(32, bytes);
    memset(bm[c], 0xFF, bytes);
  }

  std::ifstream fin(cmd_path);
  if (!fin.is_open()) { fprintf(stderr, "cannot open %s\n", cmd_path); return 2; }
  for (int q = 0; q < max_queries; q++) {
    std::vector<std::vector<CODE>> tl(ncols), tr(ncols);
    std::vector<std::string> cmd(ncols);
    bool done = false;
    for (int c = 0; c < ncols; c++) {
      std::string input;
      if (!std::getline(fin, input)) { done = true; break; }
      std::vector<std::string> cmds = stringSplit(input, ' ');
      if (cmds.empty() || cmds[0] == "exit") { done = true; break; }
      cmd[c] = cmds[0];
      if (cmds.size() > 1) tl[c] = get_target_numbers(cmds[1]);
      if (cmds.size() > 2) tr[c] = get_target_numbers(cmds[2]);
    }
    if (done) break;

    double best = 1e300;
    for (int r = 0; r < repeats; r++) {
      auto s = std::chrono::steady_clock::now();
      for (int c = 0; c < ncols; c++) {
        for (size_t pi = 0; pi < tl[c].size(); pi++) {
          CODE t1 = tl[c][pi], t2 = 0;
          if (!tr[c].empty()) t2 = tr[c][pi];
          if (cmd[c] == "bt" && t1 > t2) std::swap(t1, t2);
          run_op(bindexs[c], bm[c], cmd[c], t1, t2);
        }
      }
      for (int c = 1; c < ncols; c++) and_merge(bm[0], bm[c]);
      double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s).count();
      if (ms < best) best = ms;
    }

    const bool check = q < checked;
    uint64_t a = count_bits(bm[0], kN);
    long long b = -1;
    int equal = -1;
    if (check) {
      for (int c = 0; c < ncols; c++) memset(chk[c], 0, bytes);
      for (int c = 0; c < ncols; c++)
        raw_scan_entry(&tl[c], &tr[c], cmd[c], bindexs[c], chk[c], chk[0], data[c]);
      b = (long long)count_bits(chk[0], kN);
      equal = 1;
      for (int i = 0; i < kN && equal; i++)
        if (((bm[0][i >> 5] ^ chk[0][i >> 5]) >> (31 - (i & 31))) & 1u) equal = 0;
    }
    printf("query %d bindex_hits %llu raw_hits %lld equal %d scan_ms %.4f\n", q, (unsigned long long)a, b, equal,
           best);
    fflush(stdout);
    if (out_dir[0]) {
      char fn[8192];
      snprintf(fn, sizeof fn, "%s/q%05d_bindex.bin", out_dir, q);
      FILE *o = fopen(fn, "wb");
      if (o) { fwrite(bm[0], sizeof(BITS), W, o); fclose(o); }
      if (check) {
        snprintf(fn, sizeof fn, "%s/q%05d_raw.bin", out_dir, q);
        o = fopen(fn, "wb");
        if (o) { fwrite(chk[0], sizeof(BITS), W, o); fclose(o); }
      }
    }
  }
  return 0;
}
