// hpr_cbf.cpp — multi-threaded reader of CBF (Conic Benchmark Format) files.
//
// Follows the reference's reader (read_cbf and _read_cbf_mmap,
// src/utils/cbf_io.jl:1133-1455, with _cbf_prepare_layout 493-634) and
// returns the inputs of build_from_SOCP_data in its layout:
//   * constraint rows: equalities (L=), inequalities (L+, and L- negated so
//     every inequality reads A x >= rhs), then second-order-cone rows (Q);
//     free rows (F) are dropped;
//   * CBF states A x + b in the cone, so rhs = -b on L=, L+ and Q rows and
//     rhs = b on (negated) L- rows;
//   * variables: linear ones first (L+ >= 0, L- <= 0, L= fixed at 0, F
//     free), then cone variables;
//   * ACOORD entries whose value is zero are skipped, duplicates are summed
//     in file order and entries that sum to zero are dropped (sparse! and
//     dropzeros!); BCOORD and OBJACOORD entries are assignments, so a later
//     entry for the same index wins; entries read before both CON and VAR
//     were seen are applied after the others, as in the reference;
//   * OBJSENSE MAX negates c and the objective offset.
// Keyword lines skip blank and '#' lines and are trimmed; the lines that
// follow a keyword are taken as they come (_cbf_next_line_bounds), and
// numbers are parsed the way the reference does (decimal integers, strtod).
//
// The ACOORD block, which carries almost all of a large file, is located
// and parsed by all threads: line terminators are counted in parallel to
// find the block's end, each thread parses the lines that start in its
// share of the block's bytes, and the CSR matrix is built by a stable
// per-thread counting sort by row followed by a per-row ordering by column.
// The result does not depend on the thread count.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/hprsocp_b200.h"

struct hpr_cbf {
  int64_t m = 0, n = 0, number_eq = 0, number_ineq = 0;
  std::vector<int32_t> rowptr, col;
  std::vector<double> val, rhs, c, l, u, AL, AU;
  std::vector<int64_t> con1, var1, con0, var0;  // cone starts + sentinel, 1- and 0-based
  double obj_constant = 0.0;
};

namespace {

thread_local std::string g_cbf_err;

struct CbfError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
[[noreturn]] void fail(const std::string& s) { throw CbfError(s); }

inline bool is_space(char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; }
inline bool is_term(char ch) { return ch == '\n' || ch == '\r'; }

struct Span {
  int64_t b = 0, e = 0;  // [b, e), terminator excluded
};

// ---- number parsing (_cbf_parse_ascii_int / _cbf_parse_ascii_float)
int64_t parse_int(const char* d, int64_t& i, int64_t e) {
  while (i < e && is_space(d[i])) ++i;
  if (i >= e) fail("Invalid CBF line: expected integer token.");
  int64_t sign = 1;
  if (d[i] == '-') {
    sign = -1;
    ++i;
  } else if (d[i] == '+') {
    ++i;
  }
  int64_t v = 0;
  bool digit = false;
  while (i < e && d[i] >= '0' && d[i] <= '9') {
    v = 10 * v + (d[i] - '0');
    digit = true;
    ++i;
  }
  if (!digit) fail("Invalid CBF line: expected integer token.");
  return sign * v;
}

// The reference calls strtod.  std::from_chars gives the same correctly
// rounded value for decimal and inf/nan tokens; what it reads differently
// (a leading '+', hexadecimal, values out of range) goes to strtod on a
// NUL-terminated copy of the rest of the line.
double parse_float(const char* d, int64_t& i, int64_t e) {
  while (i < e && is_space(d[i])) ++i;
  if (i >= e) fail("Invalid CBF line: expected floating-point token.");
  const char* p = d + i;
  const char* end = d + e;
  const char* q = (*p == '+') ? p + 1 : p;
  const char* h = (q < end && *q == '-') ? q + 1 : q;
  const bool hex = end - h >= 2 && h[0] == '0' && (h[1] == 'x' || h[1] == 'X');
  const bool two_signs = q != p && q < end && (*q == '+' || *q == '-');
  if (!hex && !two_signs) {
    double v = 0.0;
    const std::from_chars_result r = std::from_chars(q, end, v);
    if (r.ec == std::errc()) {
      i = (int64_t)(r.ptr - d);
      return v;
    }
    if (r.ec == std::errc::invalid_argument) fail("Invalid CBF line: expected floating-point token.");
  }
  const std::string tok(p, end);
  char* stop = nullptr;
  const double v = std::strtod(tok.c_str(), &stop);
  const int64_t used = (int64_t)(stop - tok.c_str());
  if (used <= 0) fail("Invalid CBF line: expected floating-point token.");
  i += used;
  return v;
}

struct Group {
  std::string cone;
  int64_t len;
};

Group parse_group(const char* d, Span s) {
  int64_t i = s.b;
  while (i < s.e && is_space(d[i])) ++i;
  if (i >= s.e) fail("Invalid CBF line: expected a cone tag and length.");
  const int64_t cb = i;
  while (i < s.e && d[i] != ' ' && d[i] != '\t') ++i;
  Group g;
  g.cone.assign(d + cb, d + i);
  g.len = parse_int(d, i, s.e);
  return g;
}

std::string strip(const std::string& s) {
  size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b])) ++b;
  while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
  return s.substr(b, e - b);
}

int worker_count(int requested) {
  if (requested > 0) return requested;
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)std::min(hc, 64u) : 1;
}

template <class F>
void parallel_for(int T, F f) {
  if (T <= 1) {
    f(0);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(T - 1);
  for (int t = 1; t < T; ++t) th.emplace_back(f, t);
  f(0);
  for (auto& x : th) x.join();
}

// ---- the layout (_cbf_prepare_layout)
struct Layout {
  int64_t m_old = 0, n = 0, rows = 0, number_eq = 0, number_ineq = 0, number_lu_x = 0;
  std::vector<int64_t> row_new;   // -1: dropped (F)
  std::vector<int8_t> a_sign, b_sign;
  std::vector<int64_t> col_new;
  std::vector<double> lb, ub;
  std::vector<int64_t> con1, var1;  // 1-based starts + sentinel
};

bool supported(const std::string& t) { return t == "L+" || t == "L-" || t == "L=" || t == "Q" || t == "F"; }

Layout prepare_layout(const std::vector<Group>& con, const std::vector<Group>& var, int64_t nconstr, int64_t nvar) {
  if (con.empty()) fail("Invalid CBF file: missing CON section.");
  if (var.empty()) fail("Invalid CBF file: missing VAR section.");
  for (const Group& g : con)
    if (!supported(g.cone)) fail("Unsupported constraint cone type " + g.cone + ".");
  for (const Group& g : var)
    if (!supported(g.cone)) fail("Unsupported variable cone type " + g.cone + ".");
  Layout L;
  int64_t m = 0, n = 0;
  for (const Group& g : con) m += g.len;
  for (const Group& g : var) n += g.len;
  if (!(nconstr == -1 || nconstr == m))
    fail("CBF CON size mismatch: declared nconstr=" + std::to_string(nconstr) + " but group sum is " +
         std::to_string(m) + ".");
  if (!(nvar == -1 || nvar == n))
    fail("CBF VAR size mismatch: declared nvar=" + std::to_string(nvar) + " but group sum is " + std::to_string(n) +
         ".");
  if (m < 0 || n < 0) fail("Invalid CBF file: negative group length.");
  std::vector<int64_t> soc_lens;
  int64_t soc_rows = 0;
  for (const Group& g : con) {
    if (g.len < 0) fail("Invalid CBF file: negative group length.");
    if (g.cone == "L=") L.number_eq += g.len;
    else if (g.cone == "L+" || g.cone == "L-") L.number_ineq += g.len;
    else if (g.cone == "Q") {
      soc_rows += g.len;
      soc_lens.push_back(g.len);
    }
  }
  L.m_old = m;
  L.n = n;
  L.rows = L.number_eq + L.number_ineq + soc_rows;
  L.row_new.assign(m, -1);
  L.a_sign.assign(m, 1);
  L.b_sign.assign(m, -1);
  int64_t eq = 0, ineq = L.number_eq, soc = L.number_eq + L.number_ineq, r0 = 0;
  for (const Group& g : con) {
    for (int64_t r = r0; r < r0 + g.len; ++r) {
      if (g.cone == "L=") L.row_new[r] = eq++;
      else if (g.cone == "L+") L.row_new[r] = ineq++;
      else if (g.cone == "L-") {
        L.row_new[r] = ineq++;
        L.a_sign[r] = -1;
        L.b_sign[r] = 1;
      } else if (g.cone == "Q") L.row_new[r] = soc++;
    }
    r0 += g.len;
  }
  int64_t soc_vars = 0;
  for (const Group& g : var) {
    if (g.len < 0) fail("Invalid CBF file: negative group length.");
    if (g.cone == "Q") soc_vars += g.len;
  }
  L.number_lu_x = n - soc_vars;
  L.lb.assign(n, 0.0);
  L.ub.assign(n, 0.0);
  L.col_new.assign(n, 0);
  L.var1.push_back(L.number_lu_x + 1);
  const double inf = std::numeric_limits<double>::infinity();
  int64_t lin = 0, sv = L.number_lu_x, c0 = 0;
  for (const Group& g : var) {
    if (g.cone == "Q") {
      for (int64_t k = c0; k < c0 + g.len; ++k) {
        L.col_new[k] = sv;
        L.lb[sv] = -inf;
        L.ub[sv] = inf;
        ++sv;
      }
      L.var1.push_back(sv + 1);
    } else {
      const double lo = (g.cone == "L+" || g.cone == "L=") ? 0.0 : -inf;
      const double hi = (g.cone == "L-" || g.cone == "L=") ? 0.0 : inf;
      for (int64_t k = c0; k < c0 + g.len; ++k) {
        L.col_new[k] = lin;
        L.lb[lin] = lo;
        L.ub[lin] = hi;
        ++lin;
      }
    }
    c0 += g.len;
  }
  L.con1.push_back(L.number_eq + L.number_ineq + 1);
  for (int64_t len : soc_lens) L.con1.push_back(L.con1.back() + len);
  return L;
}

// ---- the file and its lines
struct Text {
  const char* p = "";  // the file's bytes (mapped, or `owned`)
  int64_t n = 0;
  void* map = nullptr;
  size_t map_len = 0;
  std::vector<char> owned;
  Text() = default;
  Text(const Text&) = delete;
  Text& operator=(const Text&) = delete;
  ~Text() {
    if (map) munmap(map, map_len);
  }
  const char* d() const { return p; }

  // _cbf_next_line_bounds
  bool next_raw(int64_t& pos, Span& s) const {
    if (pos >= n) return false;
    const char* p = d();
    s.b = pos;
    while (pos < n && !is_term(p[pos])) ++pos;
    s.e = pos;
    if (pos < n && p[pos] == '\r') {
      ++pos;
      if (pos < n && p[pos] == '\n') ++pos;
    } else if (pos < n && p[pos] == '\n') {
      ++pos;
    }
    return true;
  }
  // _cbf_next_data_line
  bool next_data(int64_t& pos, Span& s) const {
    const char* p = d();
    while (next_raw(pos, s)) {
      while (s.b < s.e && is_space(p[s.b])) ++s.b;
      if (s.b >= s.e || p[s.b] == '#') continue;
      while (s.e > s.b && is_space(p[s.e - 1])) --s.e;
      return true;
    }
    return false;
  }
  bool equals(Span s, const char* lit) const {
    const size_t k = std::strlen(lit);
    return (size_t)(s.e - s.b) == k && std::memcmp(d() + s.b, lit, k) == 0;
  }
  // position just past the terminator of the line ending at or after i:
  // '\n', or '\r' not followed by '\n', ends a line
  bool ends_line(int64_t i) const {
    const char* p = d();
    return p[i] == '\n' || (p[i] == '\r' && (i + 1 >= n || p[i + 1] != '\n'));
  }
  // Start of line k after `pos` (skipping k complete lines), counting line
  // terminators in parallel windows; -1 when the file ends first.  A final
  // line without a terminator counts as a line.
  int64_t skip_lines(int64_t pos, int64_t k, int T) const {
    if (k <= 0) return pos;
    const int64_t kWindowPerThread = int64_t(8) << 20;
    int64_t need = k;
    int64_t w0 = pos;
    while (w0 < n) {
      const int64_t span = std::min<int64_t>(n - w0, (int64_t)T * kWindowPerThread);
      const int Tw = span < (int64_t(1) << 20) ? 1 : T;
      std::vector<int64_t> cnt(Tw, 0);
      auto lo = [&](int t) { return w0 + span * t / Tw; };
      parallel_for(Tw, [&](int t) {
        int64_t c = 0;
        for (int64_t i = lo(t), e = lo(t + 1); i < e; ++i) c += ends_line(i) ? 1 : 0;
        cnt[t] = c;
      });
      for (int t = 0; t < Tw; ++t) {
        if (cnt[t] < need) {
          need -= cnt[t];
          continue;
        }
        for (int64_t i = lo(t), e = lo(t + 1); i < e; ++i) {
          if (ends_line(i) && --need == 0) return i + 1;
        }
      }
      w0 += span;
    }
    // the file ended: an unterminated last line counts once
    if (need == 1 && n > 0 && !is_term(d()[n - 1]) && pos < n) return n;
    return -1;
  }
};

// A coordinate block found by the scan: lines [b, e), `count` of them.
struct Block {
  int64_t b = 0, e = 0, count = 0;
  bool ready = false;  // the layout was known when the block was read
};

// Entries of a coordinate block: index pairs (ACOORD, mapped to the new
// rows and columns) or single indices (BCOORD, OBJACOORD, as written).
struct Entries {
  std::vector<int32_t> I, J;  // ACOORD: new row and column
  std::vector<int64_t> idx;   // BCOORD / OBJACOORD: 0-based index as written
  std::vector<double> V;
};

// Parse the `count` lines of a block with all threads: thread t takes the
// lines that start in its share of the block's bytes; `line(d, span, out,
// lines)` parses one line.  The threads' entries are appended to `out` in
// file order, and the first malformed line (in file order) is reported.
template <class LineFn>
void parse_lines(const Text& tx, const Block& blk, int T, bool pairs, Entries& out, LineFn line) {
  const char* d = tx.d();
  const int64_t bytes = blk.e - blk.b;
  const int Tw = (bytes < (int64_t(1) << 20) || blk.count < 4096) ? 1 : T;
  std::vector<int64_t> start(Tw + 1);
  start[0] = blk.b;
  start[Tw] = blk.e;
  for (int t = 1; t < Tw; ++t) {
    int64_t p = blk.b + bytes * t / Tw;
    while (p < blk.e && !tx.ends_line(p - 1)) ++p;  // the next line start
    start[t] = std::max(p, start[t - 1]);
  }
  std::vector<Entries> part(Tw);  // (each thread's entries, in file order)
  std::vector<int64_t> lines(Tw, 0);
  std::vector<std::string> errs(Tw);
  parallel_for(Tw, [&](int t) {
    Entries& o = part[t];
    const int64_t est = (int64_t)((double)blk.count * (double)(start[t + 1] - start[t]) /
                                  (double)std::max<int64_t>(bytes, 1)) + 16;
    o.V.reserve(est);
    if (pairs) {
      o.I.reserve(est);
      o.J.reserve(est);
    } else {
      o.idx.reserve(est);
    }
    try {
      int64_t pos = start[t], cnt = 0;
      Span sp;
      while (pos < start[t + 1] && tx.next_raw(pos, sp)) {
        line(d, sp, o);
        ++cnt;
      }
      lines[t] = cnt;
    } catch (const CbfError& e) {
      errs[t] = e.what();
    }
  });
  for (int t = 0; t < Tw; ++t)
    if (!errs[t].empty()) fail(errs[t]);
  int64_t tot = 0;
  for (int t = 0; t < Tw; ++t) tot += lines[t];
  if (tot != blk.count) fail("Invalid CBF file: malformed coordinate block.");
  std::vector<size_t> off(Tw + 1, out.V.size());
  for (int t = 0; t < Tw; ++t) off[t + 1] = off[t] + part[t].V.size();
  out.V.resize(off[Tw]);
  if (pairs) {
    out.I.resize(off[Tw]);
    out.J.resize(off[Tw]);
  } else {
    out.idx.resize(off[Tw]);
  }
  parallel_for(Tw, [&](int t) {
    const Entries& e = part[t];
    std::copy(e.V.begin(), e.V.end(), out.V.begin() + off[t]);
    if (pairs) {
      std::copy(e.I.begin(), e.I.end(), out.I.begin() + off[t]);
      std::copy(e.J.begin(), e.J.end(), out.J.begin() + off[t]);
    } else {
      std::copy(e.idx.begin(), e.idx.end(), out.idx.begin() + off[t]);
    }
  });
}

// ACOORD lines "row col value": range-checked, mapped to the new layout;
// F rows and zero values are skipped (_read_cbf_mmap).
void parse_acoord(const Text& tx, const Block& blk, const Layout& L, int T, Entries& out) {
  parse_lines(tx, blk, T, true, out, [&L](const char* d, Span sp, Entries& o) {
    int64_t i = sp.b;
    const int64_t r = parse_int(d, i, sp.e);
    const int64_t c = parse_int(d, i, sp.e);
    const double v = parse_float(d, i, sp.e);
    if (r < 0 || r >= L.m_old || c < 0 || c >= L.n) fail("Invalid CBF file: ACOORD index out of range.");
    const int64_t rn = L.row_new[r];
    if (rn < 0) return;
    const double a = (double)L.a_sign[r] * v;
    if (a == 0.0) return;
    o.I.push_back((int32_t)rn);
    o.J.push_back((int32_t)L.col_new[c]);
    o.V.push_back(a);
  });
}

// BCOORD / OBJACOORD lines "index value", as written.
void parse_pairs(const Text& tx, const Block& blk, int T, Entries& out) {
  parse_lines(tx, blk, T, false, out, [](const char* d, Span sp, Entries& o) {
    int64_t i = sp.b;
    const int64_t k = parse_int(d, i, sp.e);
    const double v = parse_float(d, i, sp.e);
    o.idx.push_back(k);
    o.V.push_back(v);
  });
}

// sparse!(I, J, V) + dropzeros!: CSR with ascending columns, duplicates
// summed in input order, zero sums removed.
void build_csr(int64_t rows, const std::vector<int32_t>& I, const std::vector<int32_t>& J,
               const std::vector<double>& V, int T, hpr_cbf& o) {
  const int64_t nnz = (int64_t)V.size();
  int Tc = T;
  if ((double)rows * Tc * sizeof(int64_t) > 1.0e9 || nnz < (int64_t(1) << 16)) Tc = 1;
  // per-thread row counts over contiguous entry ranges (stable scatter)
  std::vector<std::vector<int64_t>> cnt(Tc, std::vector<int64_t>(rows + 1, 0));
  auto elo = [&](int t) { return nnz * t / Tc; };
  parallel_for(Tc, [&](int t) {
    for (int64_t k = elo(t); k < elo(t + 1); ++k) ++cnt[t][I[k]];
  });
  std::vector<int64_t> rs(rows + 1, 0);
  for (int64_t r = 0; r < rows; ++r) {
    int64_t s = 0;
    for (int t = 0; t < Tc; ++t) s += cnt[t][r];
    rs[r + 1] = rs[r] + s;
  }
  // offsets: row start + entries of earlier threads
  parallel_for(Tc, [&](int t) {
    const int64_t r0 = rows * t / Tc, r1 = rows * (t + 1) / Tc;
    for (int64_t r = r0; r < r1; ++r) {
      int64_t p = rs[r];
      for (int tt = 0; tt < Tc; ++tt) {
        const int64_t cn = cnt[tt][r];
        cnt[tt][r] = p;
        p += cn;
      }
    }
  });
  std::vector<int32_t> tc(nnz);
  std::vector<double> tv(nnz);
  parallel_for(Tc, [&](int t) {
    for (int64_t k = elo(t); k < elo(t + 1); ++k) {
      const int64_t p = cnt[t][I[k]]++;
      tc[p] = J[k];
      tv[p] = V[k];
    }
  });
  cnt.clear();
  // per row: stable order by column, sum duplicates left to right, drop zeros
  std::vector<int64_t> keep(rows, 0);
  parallel_for(T, [&](int t) {
    const int64_t r0 = rows * t / T, r1 = rows * (t + 1) / T;
    std::vector<std::pair<int32_t, double>> tmp;
    for (int64_t r = r0; r < r1; ++r) {
      const int64_t b = rs[r], e = rs[r + 1];
      bool sorted = true;
      for (int64_t k = b + 1; k < e && sorted; ++k) sorted = tc[k - 1] <= tc[k];
      if (!sorted && e - b <= 32) {
        // stable insertion sort of the row
        for (int64_t k = b + 1; k < e; ++k) {
          const int32_t cc = tc[k];
          const double vv = tv[k];
          int64_t j = k;
          for (; j > b && tc[j - 1] > cc; --j) {
            tc[j] = tc[j - 1];
            tv[j] = tv[j - 1];
          }
          tc[j] = cc;
          tv[j] = vv;
        }
      } else if (!sorted) {
        tmp.assign(e - b, {0, 0.0});
        for (int64_t k = b; k < e; ++k) tmp[k - b] = {tc[k], tv[k]};
        std::stable_sort(tmp.begin(), tmp.end(),
                         [](const std::pair<int32_t, double>& x, const std::pair<int32_t, double>& y) {
                           return x.first < y.first;
                         });
        for (int64_t k = b; k < e; ++k) {
          tc[k] = tmp[k - b].first;
          tv[k] = tmp[k - b].second;
        }
      }
      int64_t w = b;
      for (int64_t k = b; k < e;) {
        const int32_t cc = tc[k];
        double sum = tv[k];
        int64_t j = k + 1;
        while (j < e && tc[j] == cc) sum = sum + tv[j++];
        if (sum != 0.0) {
          tc[w] = cc;
          tv[w] = sum;
          ++w;
        }
        k = j;
      }
      keep[r] = w - b;
    }
  });
  o.rowptr.assign(rows + 1, 0);
  int64_t tot = 0;
  for (int64_t r = 0; r < rows; ++r) {
    tot += keep[r];
    if (tot > std::numeric_limits<int32_t>::max()) fail("CBF matrix has more than 2^31-1 nonzeros.");
    o.rowptr[r + 1] = (int32_t)tot;
  }
  o.col.resize(tot);
  o.val.resize(tot);
  parallel_for(T, [&](int t) {
    const int64_t r0 = rows * t / T, r1 = rows * (t + 1) / T;
    for (int64_t r = r0; r < r1; ++r) {
      std::copy(tc.begin() + rs[r], tc.begin() + rs[r] + keep[r], o.col.begin() + o.rowptr[r]);
      std::copy(tv.begin() + rs[r], tv.begin() + rs[r] + keep[r], o.val.begin() + o.rowptr[r]);
    }
  });
}

// Maps the file read-only (as the reference does); files that cannot be
// mapped are read into memory.
void read_file(const char* path, Text& tx) {
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) fail(std::string("cannot open ") + path + ": " + std::strerror(errno));
  struct stat st;
  if (::fstat(fd, &st) != 0) {
    ::close(fd);
    fail(std::string("cannot read ") + path);
  }
  const size_t sz = (size_t)st.st_size;
  if (sz > 0) {
    void* m = ::mmap(nullptr, sz, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m != MAP_FAILED) {
      ::madvise(m, sz, MADV_WILLNEED);
      tx.map = m;
      tx.map_len = sz;
      tx.p = static_cast<const char*>(m);
      tx.n = (int64_t)sz;
    } else {
      tx.owned.resize(sz);
      size_t got = 0;
      while (got < sz) {
        const ssize_t k = ::read(fd, tx.owned.data() + got, sz - got);
        if (k <= 0) break;
        got += (size_t)k;
      }
      if (got != sz) {
        ::close(fd);
        fail(std::string("cannot read ") + path);
      }
      tx.p = tx.owned.data();
      tx.n = (int64_t)sz;
    }
  }
  ::close(fd);
}

hpr_cbf* read_cbf(const char* path, int nthreads) {
  const std::string fn = path ? path : "";
  auto ends = [&](const char* s) {
    const size_t k = std::strlen(s);
    return fn.size() >= k && fn.compare(fn.size() - k, k, s) == 0;
  };
  if (!(ends(".cbf") || ends(".CBF"))) fail("Unsupported file format. Please provide a .cbf file.");
  const int T = worker_count(nthreads);
  Text tx;
  read_file(path, tx);
  const char* d = tx.d();

  std::vector<Group> con, var;
  int64_t nconstr = -1, nvar = -1;
  std::string sense = "min";
  double obj_constant = 0.0;
  bool ready = false;
  std::vector<Block> ablk, bblk, cblk;

  auto groups = [&](int64_t& pos, const char* what, std::vector<Group>& g, int64_t& total) {
    Span s;
    if (!tx.next_raw(pos, s)) fail(std::string("Invalid CBF file: unexpected EOF after ") + what + ".");
    int64_t i = s.b;
    total = parse_int(d, i, s.e);
    const int64_t ng = parse_int(d, i, s.e);
    g.assign(ng > 0 ? ng : 0, Group());
    for (int64_t j = 0; j < ng; ++j) {
      if (!tx.next_raw(pos, s)) fail(std::string("Invalid CBF file: unexpected EOF inside ") + what + ".");
      g[j] = parse_group(d, s);
    }
    if (!ready && !con.empty() && !var.empty()) ready = true;
  };
  auto block = [&](int64_t& pos, const char* what, std::vector<Block>& out) {
    Span s;
    if (!tx.next_raw(pos, s)) fail(std::string("Invalid CBF file: unexpected EOF after ") + what + ".");
    int64_t i = s.b;
    const int64_t k = parse_int(d, i, s.e);
    Block b;
    b.b = pos;
    b.count = k > 0 ? k : 0;
    b.ready = ready;
    const int64_t e = tx.skip_lines(pos, b.count, T);
    if (e < 0) fail(std::string("Invalid CBF file: unexpected EOF inside ") + what + ".");
    b.e = e;
    pos = e;
    out.push_back(b);
  };

  int64_t pos = 0;
  Span s;
  while (tx.next_data(pos, s)) {
    if (tx.equals(s, "CON")) {
      groups(pos, "CON", con, nconstr);
    } else if (tx.equals(s, "VAR")) {
      groups(pos, "VAR", var, nvar);
    } else if (tx.equals(s, "ACOORD")) {
      block(pos, "ACOORD", ablk);
    } else if (tx.equals(s, "BCOORD")) {
      block(pos, "BCOORD", bblk);
    } else if (tx.equals(s, "OBJACOORD")) {
      block(pos, "OBJACOORD", cblk);
    } else if (tx.equals(s, "OBJBCOORD")) {
      Span v;
      if (!tx.next_raw(pos, v)) fail("Invalid CBF file: unexpected EOF after OBJBCOORD.");
      int64_t i = v.b;
      obj_constant = parse_float(d, i, v.e);
    } else if (tx.equals(s, "SENSE") || tx.equals(s, "OBJSENSE")) {
      Span v;
      if (!tx.next_raw(pos, v)) fail("Invalid CBF file: unexpected EOF after objective sense section.");
      const std::string raw(d + v.b, d + v.e);
      std::string t = strip(raw);
      for (char& ch : t) ch = (char)std::tolower((unsigned char)ch);
      if (t == "min" || t == "minimize" || t == "minimise") sense = "min";
      else if (t == "max" || t == "maximize" || t == "maximise") sense = "max";
      else fail("Unsupported CBF objective sense: \"" + raw + "\".");
    } else {
      const bool psd = tx.equals(s, "DCOORD") || tx.equals(s, "HCOORD") || tx.equals(s, "hCOORD") ||
                       tx.equals(s, "PSDCON");
      const bool mat = tx.equals(s, "FCOORD") || tx.equals(s, "OBJFCOORD") || tx.equals(s, "PSDVAR");
      const bool integer = tx.equals(s, "INT");
      if (!(psd || mat || integer)) continue;
      Span v;
      if (!tx.next_raw(pos, v)) fail("Invalid CBF file: unexpected EOF after section header.");
      int64_t i = v.b;
      const int64_t k = parse_int(d, i, v.e);
      if (k != 0)
        fail(psd ? "PSD constraints are not supported."
                 : mat ? "Matrix variables are not supported." : "Integer variables are not supported.");
    }
  }
  const Layout L = prepare_layout(con, var, nconstr, nvar);

  hpr_cbf* o = new hpr_cbf();
  try {
    o->m = L.rows;
    o->n = L.n;
    o->number_eq = L.number_eq;
    o->number_ineq = L.number_ineq;
    o->l = L.lb;
    o->u = L.ub;
    o->con1 = L.con1;
    o->var1 = L.var1;
    // blocks read with the layout known come first, then the others
    auto ordered = [](const std::vector<Block>& v) {
      std::vector<Block> out;
      for (const Block& b : v)
        if (b.ready) out.push_back(b);
      for (const Block& b : v)
        if (!b.ready) out.push_back(b);
      return out;
    };
    // c and b: later entries win
    o->c.assign(L.n, 0.0);
    for (const Block& b : ordered(cblk)) {
      Entries t;
      parse_pairs(tx, b, T, t);
      for (size_t k = 0; k < t.V.size(); ++k) {
        if (t.idx[k] < 0 || t.idx[k] >= L.n) fail("Invalid CBF file: OBJACOORD index out of range.");
        o->c[L.col_new[t.idx[k]]] = t.V[k];
      }
    }
    o->rhs.assign(L.rows, 0.0);
    for (const Block& b : ordered(bblk)) {
      Entries t;
      parse_pairs(tx, b, T, t);
      for (size_t k = 0; k < t.V.size(); ++k) {
        if (t.idx[k] < 0 || t.idx[k] >= L.m_old) fail("Invalid CBF file: BCOORD index out of range.");
        const int64_t rn = L.row_new[t.idx[k]];
        if (rn >= 0) o->rhs[rn] = (double)L.b_sign[t.idx[k]] * t.V[k];
      }
    }
    // A: kept entries in order, mapped to the new rows and columns
    Entries A;
    for (const Block& b : ordered(ablk)) parse_acoord(tx, b, L, T, A);
    if (L.rows > std::numeric_limits<int32_t>::max() || L.n > std::numeric_limits<int32_t>::max())
      fail("CBF problem too large for 32-bit indices.");
    build_csr(L.rows, A.I, A.J, A.V, T, *o);
    if (sense == "max") {
      for (double& v : o->c) v = -v;
      obj_constant = -obj_constant;
    }
    o->obj_constant = obj_constant;
    // build_from_SOCP_data layout (src/utils/builders.jl:24-108)
    const double inf = std::numeric_limits<double>::infinity();
    const int64_t nlin = L.number_eq + L.number_ineq;
    o->AL.assign(L.rows, -inf);
    o->AU.assign(L.rows, inf);
    for (int64_t r = 0; r < L.number_eq; ++r) o->AL[r] = o->AU[r] = o->rhs[r];
    for (int64_t r = L.number_eq; r < nlin; ++r) o->AL[r] = o->rhs[r];
    for (int64_t v : o->con1) o->con0.push_back(v - 1);
    for (int64_t v : o->var1) o->var0.push_back(v - 1);
  } catch (...) {
    delete o;
    throw;
  }
  return o;
}

}  // namespace

extern "C" {

int hpr_cbf_read(const char* path, int nthreads, hpr_cbf** out) {
  if (!out) return HPR_E_BAD_INPUT;
  *out = nullptr;
  g_cbf_err.clear();
  try {
    *out = read_cbf(path, nthreads);
    return HPR_OK;
  } catch (const CbfError& e) {
    g_cbf_err = e.what();
    return HPR_E_BAD_INPUT;
  } catch (const std::bad_alloc&) {
    g_cbf_err = "out of host memory while reading the CBF file";
    return HPR_E_BAD_INPUT;
  } catch (const std::exception& e) {
    g_cbf_err = e.what();
    return HPR_E_BAD_INPUT;
  }
}

const char* hpr_cbf_last_error(void) { return g_cbf_err.c_str(); }

int hpr_cbf_data_get(const hpr_cbf* f, hpr_cbf_data* out) {
  if (!f || !out) return HPR_E_BAD_INPUT;
  std::memset(out, 0, sizeof(*out));
  out->m = f->m;
  out->n = f->n;
  out->number_eq = f->number_eq;
  out->number_ineq = f->number_ineq;
  out->A.nrows = f->m;
  out->A.ncols = f->n;
  out->A.nnz = (int64_t)f->val.size();
  out->A.rowptr = f->rowptr.data();
  out->A.colind = f->col.data();
  out->A.values = f->val.data();
  out->rhs = f->rhs.data();
  out->c = f->c.data();
  out->l = f->l.data();
  out->u = f->u.data();
  out->soc_con_idx = f->con1.data();
  out->n_soc_con_idx = (int64_t)f->con1.size();
  out->soc_var_idx = f->var1.data();
  out->n_soc_var_idx = (int64_t)f->var1.size();
  out->obj_constant = f->obj_constant;
  return HPR_OK;
}

int hpr_cbf_problem(const hpr_cbf* f, hpr_problem* out) {
  if (!f || !out) return HPR_E_BAD_INPUT;
  std::memset(out, 0, sizeof(*out));
  const int64_t nlin = f->number_eq + f->number_ineq;
  out->m = f->m;
  out->n = f->n;
  out->m_lin = nlin;
  out->n_box = f->var0.empty() ? f->n : f->var0[0];
  out->A.nrows = f->m;
  out->A.ncols = f->n;
  out->A.nnz = (int64_t)f->val.size();
  out->A.rowptr = f->rowptr.data();
  out->A.colind = f->col.data();
  out->A.values = f->val.data();
  out->c = f->c.data();
  out->l = f->l.data();
  out->u = f->u.data();
  out->AL = f->AL.data();
  out->AU = f->AU.data();
  out->soc_rhs = f->rhs.data() + nlin;
  out->soc_con_idx = f->con0.data();
  out->n_soc_con_idx = (int64_t)f->con0.size();
  out->soc_var_idx = f->var0.data();
  out->n_soc_var_idx = (int64_t)f->var0.size();
  out->index_base = 0;
  out->q_kind = HPR_Q_NONE;
  out->obj_constant = f->obj_constant;
  return HPR_OK;
}

void hpr_cbf_free(hpr_cbf* f) { delete f; }

}  // extern "C"
