// hpr_plan.cpp — host planner of the fused SpMV + epilogue engine.
//
// Takes the place of the reference's SOC bucket planner (configure_soc_*_
// projection_paths!, src/algorithm.jl:1914-2223), which sorts cones into
// size buckets with one kernel family each.  Here every row of a matrix side
// is covered by cone-aligned tiles of at most kNnzTile nonzeros and kRowCap
// rows, so one launch handles linear rows and cones of every size:
//   * TASK_ROWS       — consecutive linear rows, or consecutive whole cones of
//                       at most kSmallConeMax rows, finished inside the CTA;
//   * TASK_CONE_PART  — a slice of a larger cone; the warp that completes
//                       the last slice publishes the cone's norm;
//   * TASK_CONE_APPLY — the projection of 64 rows of a larger cone, queued
//                       after all other tiles;
//   * TASK_LONG_PART  — a nonzero slice of a row longer than one tile; the CTA
//                       that completes the last slice adds the partial sums in
//                       slice order and finishes the row.
// Multi-CTA work is listed first so it starts in the first wave.
#include <algorithm>
#include <climits>

#include "hpr_internal.h"

#ifndef HPR_PLAN_LPT
#define HPR_PLAN_LPT 0
#endif

namespace hpr {

namespace {

void emit_long_row(const std::vector<int32_t>& rp, int32_t r, int32_t bigslot,
                   int32_t cone, int32_t cap, Plan& plan, std::vector<Task>& out) {
  int32_t nzb = rp[r], nze = rp[r + 1];
  int32_t nparts = (nze - nzb + cap - 1) / cap;
  LongRow lr;
  lr.row = r;
  lr.nparts = nparts;
  lr.partial_base = plan.npartials;
  lr.bigcone = bigslot;
  int32_t slot = (int32_t)plan.lng.size();
  plan.lng.push_back(lr);
  plan.npartials += nparts;
  for (int32_t p = 0; p < nparts; ++p) {
    Task t{};
    t.rb = r;
    t.re = r + 1;
    t.nzb = nzb + p * cap;
    t.nze = std::min(nze, t.nzb + cap);
    t.kind = TASK_LONG_PART;
    t.ncones = 0;
    t.cone = cone;
    t.group = slot;
    t.part = p;
    out.push_back(t);
  }
}

}  // namespace

void build_plan(const std::vector<int32_t>& rp, int64_t nrows,
                const std::vector<int64_t>& cone_starts, Plan& plan, int nnz_cap) {
  const int32_t cap = (nnz_cap > 0 && nnz_cap < kNnzTile) ? nnz_cap : kNnzTile;
  plan.nrows = nrows;
  plan.tasks.clear();
  plan.big.clear();
  plan.lng.clear();
  plan.npartials = 0;
  std::vector<Task> multi;  // multi-CTA work, emitted first
  std::vector<Task> rows;
  const int64_t lin_end = cone_starts.empty() ? nrows : cone_starts[0];

  // ---- linear rows
  int64_t r = 0;
  while (r < lin_end) {
    int64_t start = r, cnt = 0, nz = 0;
    while (r < lin_end && cnt < kRowCap) {
      int64_t rn = (int64_t)rp[r + 1] - rp[r];
      if (rn > cap) break;
      if (nz + rn > cap && cnt > 0) break;
      nz += rn;
      cnt++;
      r++;
    }
    if (cnt > 0) {
      Task t{};
      t.rb = (int32_t)start;
      t.re = (int32_t)r;
      t.nzb = rp[start];
      t.nze = rp[r];
      t.kind = TASK_ROWS;
      t.ncones = 0;
      t.cone = -1;
      t.group = -1;
      rows.push_back(t);
    }
    if (r < lin_end && (int64_t)rp[r + 1] - rp[r] > cap) {
      emit_long_row(rp, (int32_t)r, -1, -1, cap, plan, multi);
      r++;
    }
  }

  // ---- cones
  int64_t ncones = cone_starts.empty() ? 0 : (int64_t)cone_starts.size() - 1;
  Task cur{};
  bool open = false;
  auto flush = [&]() {
    if (open) rows.push_back(cur);
    open = false;
  };
  for (int64_t k = 0; k < ncones; ++k) {
    int64_t a = cone_starts[k], b = cone_starts[k + 1];
    int64_t d = b - a;
    int64_t cnz = (int64_t)rp[b] - rp[a];
    bool big = d > kSmallConeMax || cnz > cap;
    if (d <= 0) continue;
    if (!big) {
      if (open && ((cur.re - cur.rb) + d > kRowCap ||
                   (int64_t)(cur.nze - cur.nzb) + cnz > cap ||
                   cur.ncones >= 32000))
        flush();
      if (!open) {
        cur = Task{};
        cur.rb = (int32_t)a;
        cur.re = (int32_t)a;
        cur.nzb = rp[a];
        cur.nze = rp[a];
        cur.kind = TASK_ROWS;
        cur.ncones = 0;
        cur.cone = (int32_t)k;
        cur.group = -1;
        open = true;
      }
      cur.re = (int32_t)b;
      cur.nze = rp[b];
      cur.ncones++;
      continue;
    }
    flush();
    int32_t slot = (int32_t)plan.big.size();
    BigCone bc;
    bc.cone = (int32_t)k;
    bc.rb = (int32_t)a;
    bc.re = (int32_t)b;
    bc.nparts = 0;
    plan.big.push_back(bc);
    int64_t q = a;
    while (q < b) {
      int64_t rn = (int64_t)rp[q + 1] - rp[q];
      if (rn > cap) {
        emit_long_row(rp, (int32_t)q, slot, (int32_t)k, cap, plan, multi);
        plan.big[slot].nparts++;
        q++;
        continue;
      }
      int64_t start = q, cnt = 0, nz = 0;
      while (q < b && cnt < kRowCap) {
        int64_t rq = (int64_t)rp[q + 1] - rp[q];
        if (rq > cap) break;
        if (nz + rq > cap && cnt > 0) break;
        nz += rq;
        cnt++;
        q++;
      }
      Task t{};
      t.rb = (int32_t)start;
      t.re = (int32_t)q;
      t.nzb = rp[start];
      t.nze = rp[q];
      t.kind = TASK_CONE_PART;
      t.ncones = 0;
      t.cone = (int32_t)k;
      t.group = slot;
      multi.push_back(t);
      plan.big[slot].nparts++;
    }
  }
  flush();
#if HPR_PLAN_LPT
  // longest first: the tiles that end a launch are the lightest ones
  std::stable_sort(rows.begin(), rows.end(),
                   [](const Task& x, const Task& y) { return (x.nze - x.nzb) > (y.nze - y.nzb); });
#endif
  plan.tasks = multi;
  plan.tasks.insert(plan.tasks.end(), rows.begin(), rows.end());
  // big cones: slice numbers, norm-share slots and the apply tiles, which
  // go last (a warp that takes one finds every slice of every cone taken)
  std::vector<int32_t> next_part(plan.big.size(), 0);
  for (Task& t : plan.tasks)
    if (t.kind == TASK_CONE_PART) t.part = next_part[t.group]++;
  for (LongRow& lr : plan.lng)
    if (lr.bigcone >= 0) lr.cpart = next_part[lr.bigcone]++;
    else lr.cpart = -1;
  plan.ncparts = 0;
  for (size_t b = 0; b < plan.big.size(); ++b) {
    BigCone& bc = plan.big[b];
    bc.part_base = plan.ncparts;
    plan.ncparts += bc.nparts;
    bc.napply = 0;
    for (int32_t r = bc.rb; r < bc.re; r += kRowCap) {
      Task t{};
      t.rb = r;
      t.re = std::min(bc.re, r + kRowCap);
      t.nzb = t.nze = rp[r];
      t.kind = TASK_CONE_APPLY;
      t.cone = bc.cone;
      t.group = (int32_t)b;
      plan.tasks.push_back(t);
      bc.napply++;
    }
  }
  build_runs(rp, plan);
}

// Run layout of every tile (TileRun): slot offsets, non-empty rows and the
// per-lane row-start descriptors.
void build_runs(const std::vector<int32_t>& rp, Plan& plan) {
  const size_t nt = plan.tasks.size();
  plan.runs.assign(nt, TileRun{});
  plan.desc.assign(nt * 32, 0u);
  int64_t slots = 0;
  for (size_t ti = 0; ti < nt; ++ti) {
    const Task& t = plan.tasks[ti];
    const int32_t nnz = t.nze - t.nzb;
    const int32_t R = (nnz + 31) / 32;
    TileRun& tr = plan.runs[ti];
    tr.sbase = (int32_t)std::min<int64_t>(slots, INT32_MAX);
    slots += 32 * (int64_t)R;
    if (t.kind == TASK_LONG_PART) {
      tr.nonempty = 1;  // one row; its runs carry no row starts
      continue;
    }
    if (t.kind == TASK_CONE_APPLY) continue;  // no nonzeros
    uint32_t heads[32] = {0};
    for (int32_t q = t.rb; q < t.re; ++q) {
      if (rp[q + 1] <= rp[q]) continue;
      tr.nonempty |= 1ull << (q - t.rb);
      const int32_t s = rp[q] - t.nzb;  // first nonzero of the row in the tile
      heads[s / R] |= 1u << (s % R);
    }
    uint32_t before = 0;
    for (int L = 0; L < 32; ++L) {
      plan.desc[ti * 32 + L] = (uint64_t)heads[L] | ((uint64_t)before << kDescOrdShift);
      before += (uint32_t)__builtin_popcount(heads[L]);
    }
  }
  plan.tslots = slots;
}

}  // namespace hpr
