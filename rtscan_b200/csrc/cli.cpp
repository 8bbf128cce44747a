// rtscan_b200_cli -- drop-in driver for the reference's GPU BinDex driver.
//
// Mirrors bindex_cuda's main() (bindex_cuda.cpp:1708-1995): read `-b`
// columns from the column file `-f`, build the indexes, then answer the
// scan_cmd file `-p` one query per group of `-b` lines, printing the
// reference's log lines ("[Time] Index Build Time", "[Time] total time",
// "[CHECK]hit a/b").  Differences: the row count is a run-time flag (`-n`,
// default: file size / (4 * ncols)) instead of the compile-time DATA_N; the
// self-check compares the chosen plan with the plain fused scan on the GPU
// (the reference re-runs its scalar filter on the host, bindex_cuda.cpp:
// 1948-1983); `-m` picks the plan (auto | scan | bindex | batch); `-o`
// writes each result bitmap to <prefix>.<query>.bin; `-e` rank-encodes the
// table first and rewrites every query (the reference's ENCODE=1 build of
// its RT driver, rtscan.cpp:1020-1024,1069-1072); `-I <prefix>` loads each
// column's index from <prefix>.<column>.bdx when present and saves it there
// after building it otherwise; `-q <n>` answers the first n queries of the
// file, or with `-y 0` generates n queries instead (the reference RT
// driver's flags, rtscan.cpp:939-958,798-865): `-g 1` (default) range
// queries `lt (i+1)*span` on every column, `-g 0` point queries
// `eq (i+1)*span`, span = (2^32 - 1) / (n + 1).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "rtscan_b200.h"

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static int die(rts_ctx *ctx, const char *what) {
  fprintf(stderr, "[ERROR] %s: %s\n", what, rts_last_error(ctx));
  return 1;
}

static uint64_t popcount_host(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b, uint64_t *true_hit) {
  uint64_t total = 0, th = 0;
  for (size_t i = 0; i < a.size(); i++) {
    total += (uint64_t)__builtin_popcount(a[i]);
    th += (uint64_t)__builtin_popcount(a[i] & b[i]);
  }
  *true_hit = th;
  return total;
}

int main(int argc, char **argv) {
  const char *data = nullptr, *cmd_path = "test/scan_cmd.txt", *out_prefix = nullptr, *mode = "auto";
  const char *index_prefix = nullptr;
  bool encode = false, read_queries = true, range_queries = true;
  int max_queries = -1;
  int ncols = 1, K = 128, device = 0;
  uint64_t nrows = 0;
  bool check = true;
  int opt;
  while ((opt = getopt(argc, argv, "hf:b:p:n:K:m:o:d:xeI:q:y:g:")) != -1) {
    switch (opt) {
      case 'h':
        printf("Usage: %s -f <column-file> -b <ncols> -p <scan-cmd-file> [-n <rows>] [-K <areas>]\n"
               "          [-m auto|scan|bindex|batch] [-o <bitmap-prefix>] [-d <device>] [-x (no check)]\n"
               "          [-e (rank-encode the table)] [-I <index-file-prefix>]\n"
               "          [-q <queries>] [-y 0 (generate the queries)] [-g 1|0 (range|point queries)]\n",
               argv[0]);
        return 0;
      case 'f': data = optarg; break;
      case 'b': ncols = atoi(optarg); break;
      case 'p': cmd_path = optarg; break;
      case 'n': nrows = strtoull(optarg, nullptr, 10); break;
      case 'K': K = atoi(optarg); break;
      case 'm': mode = optarg; break;
      case 'o': out_prefix = optarg; break;
      case 'd': device = atoi(optarg); break;
      case 'x': check = false; break;
      case 'e': encode = true; break;
      case 'I': index_prefix = optarg; break;
      case 'q': max_queries = atoi(optarg); break;
      case 'y': read_queries = atoi(optarg) != 0; break;
      case 'g': range_queries = atoi(optarg) != 0; break;
      default: fprintf(stderr, "see -h for the options\n"); return 2;  // getopt named the bad option
    }
  }
  if (!data || ncols < 1) {
    fprintf(stderr, "need -f <column-file> and -b <ncols>\n");
    return 2;
  }
  // argument errors before any device work
  if (strcmp(mode, "auto") && strcmp(mode, "scan") && strcmp(mode, "bindex") && strcmp(mode, "batch")) {
    fprintf(stderr, "Error: unknown mode %s (auto, scan, bindex or batch)\n", mode);
    return 2;
  }
  if (!read_queries && max_queries < 1) {
    fprintf(stderr, "-y 0 needs -q <queries>\n");
    return 2;
  }
  if (read_queries && access(cmd_path, R_OK) != 0) {
    fprintf(stderr, "Fail to open scan_cmd file %s\n", cmd_path);
    return 1;
  }
  rts_ctx *ctx = nullptr;
  if (rts_open(device, &ctx) != RTS_OK) return die(nullptr, "open");
  size_t free0 = 0, free1 = 0, total = 0;
  cudaMemGetInfo(&free0, &total);
  if (rts_load_file(ctx, data, ncols, nrows) != RTS_OK) return die(ctx, "load");
  cudaMemGetInfo(&free1, &total);
  printf("[Mem] columns: %.1f MB used\n", (double)(free0 - free1) / 1e6);
  const uint64_t n = rts_nrows(ctx), words = rts_bitmap_words(n);
  printf("N = %llu\n", (unsigned long long)n);
  if (encode) {
    const double te = now_ms();
    if (rts_encode_table(ctx, 0, (uint32_t)std::min<uint64_t>(n, 0xFFFFFFFFull)) != RTS_OK) return die(ctx, "encode");
    printf("[Time] Encode Time: %.3f ms\n", now_ms() - te);
  }
  const bool want_index = !strcmp(mode, "auto") || !strcmp(mode, "bindex");
  double t0 = now_ms();
  if (want_index)
    for (int c = 0; c < ncols; c++) {
      const std::string fn = index_prefix ? std::string(index_prefix) + "." + std::to_string(c) + ".bdx" : "";
      if (index_prefix && access(fn.c_str(), R_OK) == 0) {
        if (rts_load_bindex(ctx, c, fn.c_str()) != RTS_OK) return die(ctx, "load bindex");
        continue;
      }
      if (rts_build_bindex(ctx, c, K) != RTS_OK) return die(ctx, "build bindex");
      if (index_prefix && rts_save_bindex(ctx, c, fn.c_str()) != RTS_OK) return die(ctx, "save bindex");
    }
  printf("[Time] Index Build Time: %.3f ms\n", now_ms() - t0);
  {
    size_t free2 = 0;
    cudaMemGetInfo(&free2, &total);
    printf("[Mem] indexes: %.1f MB used\n", (double)(free1 - free2) / 1e6);
  }

  std::string text;
  if (read_queries) {
    FILE *fp = fopen(cmd_path, "rb");
    if (!fp) {
      fprintf(stderr, "Fail to open scan_cmd file %s\n", cmd_path);
      return 1;
    }
    char buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, r);
    fclose(fp);
  } else {  // max_queries >= 1, checked above
    const uint32_t span = 0xFFFFFFFFu / (uint32_t)(max_queries + 1);
    for (int i = 0; i < max_queries; i++)
      for (int c = 0; c < ncols; c++)
        text += std::string(range_queries ? "lt " : "eq ") + std::to_string((uint64_t)(i + 1) * span) + "\n";
    text += "exit\n";
  }
  rts_qset *qs = nullptr;
  if (rts_parse_scan_cmd(text.data(), text.size(), ncols, &qs) != RTS_OK) return die(nullptr, "scan_cmd");
  const int nq = max_queries >= 0 ? std::min(max_queries, (int)rts_qset_size(qs)) : (int)rts_qset_size(qs);

  uint32_t *d_bm = nullptr, *d_chk = nullptr;
  uint64_t *d_cnt = nullptr;
  if (cudaMalloc(&d_bm, std::max<uint64_t>(words, 1) * 4) != cudaSuccess ||
      cudaMalloc(&d_chk, std::max<uint64_t>(words, 1) * 4) != cudaSuccess || cudaMalloc(&d_cnt, 16) != cudaSuccess) {
    fprintf(stderr, "[ERROR] device allocation failed\n");
    return 1;
  }
  std::vector<uint32_t> host(words), hchk(words);
  cudaStream_t s = nullptr;
  for (int q = 0; q < nq; q++) {
    const rts_term *terms;
    int32_t nt, empty;
    rts_qset_query(qs, q, &terms, &nt, &empty);
    std::vector<rts_term> coded(nt);
    if (encode && nt > 0) {
      if (rts_encode_terms(ctx, terms, nt, coded.data()) != RTS_OK) return die(ctx, "encode query");
      terms = coded.data();
    }
    for (int c = 0; c < ncols; c++) {
      int32_t op;
      uint32_t t1, t2;
      rts_qset_line(qs, q, c, &op, &t1, &t2);
      static const char *names[] = {"eq", "lt", "gt", "le", "ge", "bt"};
      if (op == RTS_OP_BT) printf("input %s %u %u (%d/%d)\n", names[op], t1, t2, c + 1, ncols);
      else printf("input %s %u (%d/%d)\n", names[op], t1, c + 1, ncols);
    }
    cudaDeviceSynchronize();
    const double ts = now_ms();
    rts_status st;
    if (!strcmp(mode, "scan")) {
      st = rts_scan_async(ctx, terms, nt, d_bm, d_cnt, s);
    } else if (!strcmp(mode, "batch")) {
      const int32_t off[2] = {0, nt};
      st = rts_scan_batch_async(ctx, terms, off, 1, d_bm, words, d_cnt, s);
    } else {
      st = rts_bindex_scan_async(ctx, terms, nt, d_bm, d_cnt, s);
    }
    if (st != RTS_OK) return die(ctx, "scan");
    cudaDeviceSynchronize();
    const double total = now_ms() - ts;
    const double td = now_ms();
    cudaMemcpy(host.data(), d_bm, words * 4, cudaMemcpyDeviceToHost);
    uint64_t count = 0;
    cudaMemcpy(&count, d_cnt, 8, cudaMemcpyDeviceToHost);
    const double d2h = now_ms() - td;
    printf("\n###########   Time  ##########\n[Time] total time: %.4f ms\n[Time] result transfer: %.4f ms\n"
           "##############################\n\n",
           total, d2h);
    if (check) {
      if (rts_scan_async(ctx, terms, nt, d_chk, d_cnt + 1, s) != RTS_OK) return die(ctx, "check scan");
      cudaMemcpy(hchk.data(), d_chk, words * 4, cudaMemcpyDeviceToHost);
      uint64_t true_hit = 0;
      const uint64_t total_hit = popcount_host(hchk, host, &true_hit);
      bool same = hchk == host;
      if (!same) printf("[ERROR] check error: the plan's bitmap differs from the plain scan\n");
      printf("[CHECK]hit %llu/%llu\n", (unsigned long long)true_hit, (unsigned long long)total_hit);
    }
    printf("[RESULT] query %d count %llu\n", q, (unsigned long long)count);
    if (out_prefix) {
      std::string fn = std::string(out_prefix) + "." + std::to_string(q) + ".bin";
      FILE *o = fopen(fn.c_str(), "wb");
      if (o) {
        fwrite(host.data(), 4, words, o);
        fclose(o);
      }
    }
  }
  rts_qset_free(qs);
  cudaFree(d_bm);
  cudaFree(d_chk);
  cudaFree(d_cnt);
  rts_close(ctx);
  return 0;
}
