// scan_cmd parser and operator lowering.
//
// Format (bindex.cpp:2165-2189, bindex_cuda.cpp:1834-1854, rtscan.cpp:992-1035;
// fixtures test/scan_cmd_*.txt): `ncols` consecutive lines form one
// conjunctive query, line c applying to column c.  A line is
// `<op> <t1>[,<t1>...] [<t2>[,<t2>...]]` with op in {lt,le,gt,ge,eq,bt}; a line
// whose first token is `exit` ends the list and anything after it (the
// fixtures keep free-form notes there) is ignored.  Numbers go through
// strtod and the reference's (CODE) conversion (get_target_numbers,
// bindex.cpp:1840-1849): truncation toward zero, then the low 32 bits.
//
// Where the reference's behaviour is undefined the parser reports an error
// instead: unknown operators (the reference skips them), a missing target,
// a second target on an operator other than bt (the reference asserts,
// bindex.cpp:2201), blank lines inside a query, and non-numeric targets
// (stod throws).  Runs of spaces or tabs separate tokens, and a trailing
// carriage return is ignored.  A comma list on a line expands the query
// into one query per list position; lists of length one broadcast.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <memory>
#include <new>
#include <string>
#include <vector>

#include "rts_internal.h"

struct rts_qset {
  struct Line {
    int32_t op;
    uint32_t t1, t2;
  };
  struct Query {
    std::vector<rts_term> terms;
    std::vector<Line> lines;
    int32_t empty = 0;
  };
  std::vector<Query> queries;
};

namespace {

int op_code(const std::string &s) {
  if (s == "eq") return RTS_OP_EQ;
  if (s == "lt") return RTS_OP_LT;
  if (s == "gt") return RTS_OP_GT;
  if (s == "le") return RTS_OP_LE;
  if (s == "ge") return RTS_OP_GE;
  if (s == "bt") return RTS_OP_BT;
  return -1;
}

std::vector<std::string> split_ws(const std::string &line) {
  std::vector<std::string> out;
  size_t i = 0, n = line.size();
  while (i < n) {
    while (i < n && (line[i] == ' ' || line[i] == '\t')) i++;
    size_t j = i;
    while (j < n && line[j] != ' ' && line[j] != '\t') j++;
    if (j > i) out.push_back(line.substr(i, j - i));
    i = j;
  }
  return out;
}

// (CODE)stod(v) as x86-64 g++ compiles it.
bool parse_number(const std::string &tok, uint32_t *out) {
  if (tok.empty()) return false;
  const char *s = tok.c_str();
  char *end = nullptr;
  double d = strtod(s, &end);
  if (end == s || !isfinite(d) || fabs(d) >= 9.2e18) return false;
  *out = (uint32_t)(int64_t)d;
  return true;
}

bool parse_list(const std::string &tok, std::vector<uint32_t> *out) {
  size_t start = 0;
  while (true) {
    size_t comma = tok.find(',', start);
    std::string item = tok.substr(start, comma == std::string::npos ? std::string::npos : comma - start);
    uint32_t v;
    if (!parse_number(item, &v)) return false;
    out->push_back(v);
    if (comma == std::string::npos) break;
    start = comma + 1;
  }
  return !out->empty();
}

struct ParsedLine {
  int op;
  std::vector<uint32_t> t1, t2;
};

}  // namespace

namespace {

rts_status parse_scan_cmd(const char *text, uint64_t len, int32_t ncols, rts_qset **out) {
  std::unique_ptr<rts_qset> owner(new (std::nothrow) rts_qset());
  if (!owner) return rts::set_thread_error(RTS_ERR_NOMEM, "scan_cmd: host allocation failed");
  rts_qset *qs = owner.get();
  std::vector<ParsedLine> pending;
  uint64_t pos = 0;
  int lineno = 0;
  auto error = [&](const std::string &m) {
    return rts::set_thread_error(RTS_ERR_PARSE, "scan_cmd line " + std::to_string(lineno) + ": " + m);
  };
  while (pos < len) {
    uint64_t e = pos;
    while (e < len && text[e] != '\n') e++;
    std::string line(text + pos, text + e);
    pos = e + 1;
    lineno++;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::vector<std::string> tok = split_ws(line);
    if (!tok.empty() && tok[0] == "exit") break;
    if (tok.empty()) {
      if (pending.empty()) continue;  // blank lines between queries are harmless
      return error("blank line inside a query");
    }
    ParsedLine pl;
    pl.op = op_code(tok[0]);
    if (pl.op < 0) return error("unknown operator '" + tok[0] + "'");
    if (tok.size() < 2) return error("operator '" + tok[0] + "' has no target");
    if (!parse_list(tok[1], &pl.t1)) return error("bad target '" + tok[1] + "'");
    if (pl.op == RTS_OP_BT) {
      if (tok.size() < 3) return error("bt needs two targets");
      if (!parse_list(tok[2], &pl.t2)) return error("bad target '" + tok[2] + "'");
      if (pl.t2.size() != pl.t1.size()) return error("bt target lists differ in length");
      if (tok.size() > 3) return error("too many tokens");
    } else if (tok.size() > 2) {
      return error("only bt takes a second target");
    }
    pending.push_back(std::move(pl));
    if ((int)pending.size() == ncols) {
      size_t L = 1;
      for (auto &p : pending) {
        if (p.t1.size() == 1) continue;
        if (L != 1 && p.t1.size() != L) return error("target lists of one query differ in length");
        L = p.t1.size();
      }
      for (size_t k = 0; k < L; k++) {
        rts_qset::Query q;
        for (int c = 0; c < ncols; c++) {
          const ParsedLine &p = pending[c];
          size_t idx = p.t1.size() == 1 ? 0 : k;
          uint32_t t1 = p.t1[idx], t2 = p.op == RTS_OP_BT ? p.t2[idx] : 0;
          q.lines.push_back({p.op, t1, t2});
          uint32_t lo, hi;
          int32_t ne;
          rts_lower_op(p.op, t1, t2, &lo, &hi, &ne);
          if (!ne) q.empty = 1;
          q.terms.push_back({c, lo, hi});
        }
        qs->queries.push_back(std::move(q));
      }
      pending.clear();
    }
  }
  *out = owner.release();
  return RTS_OK;
}

}  // namespace

extern "C" {

rts_status rts_parse_scan_cmd(const char *text, uint64_t len, int32_t ncols, rts_qset **out) {
  if (!out || (!text && len) || ncols < 1) return rts::set_thread_error(RTS_ERR_ARG, "bad arguments");
  *out = nullptr;
  try {  // no exception crosses the C boundary
    return parse_scan_cmd(text, len, ncols, out);
  } catch (const std::bad_alloc &) {
    return rts::set_thread_error(RTS_ERR_NOMEM, "scan_cmd: host allocation failed");
  }
}

int32_t rts_qset_size(const rts_qset *qs) { return qs ? (int32_t)qs->queries.size() : 0; }

rts_status rts_qset_query(const rts_qset *qs, int32_t i, const rts_term **terms, int32_t *nterms, int32_t *empty) {
  if (!qs || i < 0 || i >= (int)qs->queries.size() || !terms || !nterms) return RTS_ERR_ARG;
  const auto &q = qs->queries[i];
  *terms = q.terms.data();
  *nterms = (int32_t)q.terms.size();
  if (empty) *empty = q.empty;
  return RTS_OK;
}

rts_status rts_qset_line(const rts_qset *qs, int32_t i, int32_t c, int32_t *op, uint32_t *t1, uint32_t *t2) {
  if (!qs || i < 0 || i >= (int)qs->queries.size()) return RTS_ERR_ARG;
  const auto &q = qs->queries[i];
  if (c < 0 || c >= (int)q.lines.size()) return RTS_ERR_ARG;
  if (op) *op = q.lines[c].op;
  if (t1) *t1 = q.lines[c].t1;
  if (t2) *t2 = q.lines[c].t2;
  return RTS_OK;
}

void rts_qset_free(rts_qset *qs) { delete qs; }

}  // extern "C"
