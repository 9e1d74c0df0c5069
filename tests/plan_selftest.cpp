// Self-test of the engine's tile planner (hpr-socp_b200/csrc/hpr_plan.cpp),
// built on the host with the planner's own source: random row pointers and
// cone structures, every plan checked against the invariants the engine
// relies on.  Prints "ok <plans checked>" or the first violation and exits
// non-zero.
//
//   plan_selftest SEED COUNT
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../hpr-socp_b200/csrc/hpr_internal.h"

using hpr::BigCone;
using hpr::LongRow;
using hpr::Plan;
using hpr::Task;

namespace {

int g_fail = 0;
#define CHECK(cond, ...)                                        \
  do {                                                          \
    if (!(cond)) {                                              \
      std::printf("FAIL %s:%d: %s | ", __FILE__, __LINE__, #cond); \
      std::printf(__VA_ARGS__);                                 \
      std::printf("\n");                                        \
      g_fail = 1;                                               \
      return false;                                             \
    }                                                           \
  } while (0)

struct Case {
  std::vector<int32_t> rp;
  std::vector<int64_t> cones;  // first row of every cone + end sentinel (empty: no cones)
  int64_t nrows = 0;
  int cap = 0;
};

// row lengths: mostly short (lognormal, some empty), a few longer than a tile
Case make_case(std::mt19937_64& g) {
  Case c;
  std::uniform_int_distribution<int> nlin(0, 400), ncone(0, 60), pick(0, 99);
  std::lognormal_distribution<double> len(2.0, 1.0);
  const int lin = nlin(g);
  std::vector<int64_t> dims;
  const int k = ncone(g);
  for (int i = 0; i < k; ++i) {
    const int p = pick(g);
    // cones of 1..8 rows, tens of rows, or more than one tile's rows
    dims.push_back(p < 60 ? 1 + p % 8 : (p < 90 ? 10 + p : 65 + (p * 37) % 300));
  }
  c.nrows = lin;
  for (int64_t d : dims) c.nrows += d;
  c.rp.assign(c.nrows + 1, 0);
  for (int64_t r = 0; r < c.nrows; ++r) {
    int64_t n = (int64_t)len(g);
    const int p = pick(g);
    if (p < 8) n = 0;                       // empty row
    else if (p < 10) n = 1500 + 97 * p;     // longer than any tile
    c.rp[r + 1] = c.rp[r] + (int32_t)n;
  }
  if (!dims.empty()) {
    int64_t s = lin;
    for (int64_t d : dims) {
      c.cones.push_back(s);
      s += d;
    }
    c.cones.push_back(s);
  }
  const int caps[] = {0, 0, 256, 704};
  c.cap = caps[pick(g) % 4];
  return c;
}

bool check_plan(const Case& c, const Plan& p) {
  const int32_t cap = (c.cap > 0 && c.cap < hpr::kNnzTile) ? c.cap : hpr::kNnzTile;
  const int64_t lin_end = c.cones.empty() ? c.nrows : c.cones[0];
  const size_t nt = p.tasks.size();
  CHECK(p.runs.size() == nt && p.desc.size() == nt * 32, "run arrays %zu %zu", p.runs.size(), p.desc.size());
  std::vector<int> owner(c.nrows, 0);  // how many tiles or long rows own each row
  bool seen_apply = false;
  int64_t slots = 0;
  for (size_t ti = 0; ti < nt; ++ti) {
    const Task& t = p.tasks[ti];
    const int32_t nnz = t.nze - t.nzb;
    const int32_t R = (nnz + 31) / 32;
    CHECK(p.runs[ti].sbase == slots, "tile %zu sbase %d want %lld", ti, p.runs[ti].sbase, (long long)slots);
    slots += 32 * (int64_t)R;
    if (t.kind == hpr::TASK_CONE_APPLY) {
      seen_apply = true;
      CHECK(nnz == 0 && t.re > t.rb && t.re - t.rb <= hpr::kRowCap, "apply tile %zu", ti);
      continue;
    }
    CHECK(!seen_apply, "tile %zu of kind %d after an apply tile", ti, (int)t.kind);
    CHECK(nnz >= 0 && nnz <= cap, "tile %zu has %d nonzeros (cap %d)", ti, nnz, cap);
    if (t.kind == hpr::TASK_LONG_PART) {
      CHECK(t.re == t.rb + 1 && t.nzb >= c.rp[t.rb] && t.nze <= c.rp[t.rb + 1] && nnz > 0, "long slice %zu", ti);
      CHECK(p.runs[ti].nonempty == 1, "long slice %zu nonempty", ti);
      continue;
    }
    CHECK(t.re > t.rb && t.re - t.rb <= hpr::kRowCap, "tile %zu rows %d..%d", ti, t.rb, t.re);
    CHECK(t.nzb == c.rp[t.rb] && t.nze == c.rp[t.re], "tile %zu nonzero range", ti);
    // linear tiles stay linear, cone tiles hold cone rows only
    CHECK((t.re <= lin_end) || (t.rb >= lin_end), "tile %zu mixes linear and cone rows", ti);
    for (int32_t q = t.rb; q < t.re; ++q) owner[q]++;
    // run layout: row starts, ordinals and the non-empty mask
    uint64_t mask = 0;
    uint32_t heads[32] = {0};
    for (int32_t q = t.rb; q < t.re; ++q) {
      if (c.rp[q + 1] <= c.rp[q]) continue;
      mask |= 1ull << (q - t.rb);
      const int32_t s = c.rp[q] - t.nzb;
      heads[s / R] |= 1u << (s % R);
    }
    CHECK(p.runs[ti].nonempty == mask, "tile %zu nonempty mask", ti);
    uint32_t before = 0;
    for (int L = 0; L < 32; ++L) {
      const uint64_t d = p.desc[ti * 32 + L];
      CHECK((uint32_t)d == heads[L], "tile %zu lane %d row starts", ti, L);
      CHECK((uint32_t)(d >> hpr::kDescOrdShift) == before, "tile %zu lane %d ordinal", ti, L);
      CHECK(R == 0 || heads[L] >> (R - 1) >> 1 == 0, "tile %zu lane %d start bit past the run", ti, L);
      before += (uint32_t)__builtin_popcount(heads[L]);
    }
  }
  CHECK(slots == p.tslots, "tslots %lld want %lld", (long long)p.tslots, (long long)slots);
  // long rows: their slices cover the row in order
  int32_t parts_total = 0;
  for (size_t s = 0; s < p.lng.size(); ++s) {
    const LongRow& lr = p.lng[s];
    owner[lr.row]++;
    int32_t cnt = 0, at = c.rp[lr.row];
    for (size_t ti = 0; ti < nt; ++ti) {
      const Task& t = p.tasks[ti];
      if (t.kind != hpr::TASK_LONG_PART || t.group != (int32_t)s) continue;
      CHECK(t.part == cnt && t.nzb == at, "long row %zu slice %d", s, cnt);
      at = t.nze;
      cnt++;
    }
    CHECK(cnt == lr.nparts && at == c.rp[lr.row + 1], "long row %zu covered by %d of %d", s, cnt, lr.nparts);
    CHECK(lr.partial_base == parts_total, "long row %zu partial base", s);
    parts_total += lr.nparts;
    CHECK(c.rp[lr.row + 1] - c.rp[lr.row] > cap, "long row %zu is not longer than a tile", s);
  }
  CHECK(parts_total == p.npartials, "partials %d want %d", p.npartials, parts_total);
  for (int64_t r = 0; r < c.nrows; ++r) CHECK(owner[r] == 1, "row %lld owned %d times", (long long)r, owner[r]);
  // small cones whole inside one tile; big cones sliced, sliced parts numbered
  std::vector<int64_t> cone_of(c.nrows, -1);
  for (size_t k = 0; k + 1 < c.cones.size(); ++k)
    for (int64_t r = c.cones[k]; r < c.cones[k + 1]; ++r) cone_of[r] = (int64_t)k;
  int32_t cparts = 0;
  for (size_t b = 0; b < p.big.size(); ++b) {
    const BigCone& bc = p.big[b];
    CHECK(bc.rb == c.cones[bc.cone] && bc.re == c.cones[bc.cone + 1], "big cone %zu bounds", b);
    CHECK(bc.part_base == cparts, "big cone %zu part base", b);
    cparts += bc.nparts;
    std::vector<int> seen(bc.nparts, 0);
    int32_t apply = 0, covered = 0;
    for (const Task& t : p.tasks) {
      if (t.group != (int32_t)b) continue;
      if (t.kind == hpr::TASK_CONE_PART) {
        CHECK(t.part >= 0 && t.part < bc.nparts, "big cone %zu part %d", b, t.part);
        seen[t.part]++;
        covered += t.re - t.rb;
      } else if (t.kind == hpr::TASK_CONE_APPLY) {
        CHECK(t.rb == bc.rb + apply * hpr::kRowCap, "big cone %zu apply tile %d", b, apply);
        apply++;
      }
    }
    for (const LongRow& lr : p.lng)
      if (lr.bigcone == (int32_t)b) {
        CHECK(lr.cpart >= 0 && lr.cpart < bc.nparts, "big cone %zu long part", b);
        seen[lr.cpart]++;
        covered++;
      }
    for (int32_t q = 0; q < bc.nparts; ++q) CHECK(seen[q] == 1, "big cone %zu part %d seen %d", b, q, seen[q]);
    CHECK(covered == bc.re - bc.rb, "big cone %zu rows covered %d", b, covered);
    CHECK(apply == bc.napply && apply == (bc.re - bc.rb + hpr::kRowCap - 1) / hpr::kRowCap, "big cone %zu apply", b);
  }
  CHECK(cparts == p.ncparts, "norm shares %d want %d", p.ncparts, cparts);
  for (const Task& t : p.tasks) {
    if (t.kind != hpr::TASK_ROWS || t.cone < 0) continue;
    // whole cones only: the tile starts and ends on cone boundaries
    CHECK(cone_of[t.rb] == t.cone && c.cones[t.cone] == t.rb, "cone tile starts inside a cone");
    CHECK(t.re == c.nrows || cone_of[t.re] != cone_of[t.re - 1], "cone tile ends inside a cone");
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  const unsigned long long seed = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1;
  const int count = argc > 2 ? std::atoi(argv[2]) : 200;
  std::mt19937_64 g(seed);
  for (int i = 0; i < count; ++i) {
    const Case c = make_case(g);
    Plan p;
    hpr::build_plan(c.rp, c.nrows, c.cones, p, c.cap);
    if (!check_plan(c, p)) {
      std::printf("case %d (rows %lld, cones %zu, cap %d)\n", i, (long long)c.nrows,
                  c.cones.empty() ? 0 : c.cones.size() - 1, c.cap);
      return 1;
    }
  }
  std::printf("ok %d\n", count);
  return g_fail;
}
