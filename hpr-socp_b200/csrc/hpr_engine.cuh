// hpr_engine.cuh — the fused CSR SpMV + epilogue engine.
//
// One launch computes v = M * xin for every row of a matrix side and hands
// each result to an epilogue functor, so intermediate vectors (A'y, A x_hat,
// z_raw, s_raw) never reach HBM.  Work comes from the host planner
// (hpr_plan.cpp) as cone-aligned warp tiles of at most kNnzTile nonzeros and
// kRowCap rows, stored in the run layout (TileRun, hpr_internal.h): a tile's
// nonzeros cut into 32 contiguous runs, lane-interleaved.
//
// Every warp works on its own tiles with no CTA-wide synchronisation, so the
// SM's 24 resident warps hide each other's memory latency.  Persistent
// warps take their first tile by warp index (plans without split cones) and
// the rest from an atomic counter; per tile a warp
//   1. streams its run's column indices and values with coalesced
//      evict-first loads, gathers xin through L2 (ld.global.cg) and adds the
//      products of each row inside the run in column order in a register,
//      closing a row's sum into a shared-memory slot at the next row start;
//   2. adds the parts of rows that span runs with a fixed-order segmented
//      scan over the lanes, and hands each row's sum to the lane that owns
//      the row (two rows per lane);
//   3. requests the rows' epilogue inputs and runs the epilogue per row
//      (linear rows / boxed variables) or per cone (one lane per cone
//      computes ||tail||_2 serially, then one lane per row projects).  Rows
//      longer than one tile are split over several tiles, and the warp that
//      completes the last slice (atomic arrival counter, no waiting) finishes
//      them.  Cones larger than one tile are split into slices that store
//      their shares of the norm; the last slice publishes the norm and apply
//      tiles, queued after every other tile, project the rows (a bounded wait
//      for the published norm);
//   4. reduces optional scalar reductions in a fixed order and writes one
//      slot per tile, so results do not depend on scheduling.
// The last CTA to finish resets the tile counter and may advance the
// Halpern counter `inner`, so a whole iteration runs from device-resident
// scalars and can be captured in a CUDA graph.
#pragma once

#include "hpr_internal.h"

#include <type_traits>

namespace hpr {

struct Red {
  double v[kMaxRed];
};

__device__ __forceinline__ double nanmax(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return a > b ? a : b;
}
// std::max / std::min semantics (the oracle uses the same)
__device__ __forceinline__ double cmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double cmin(double a, double b) { return (b < a) ? b : a; }

template <int NRED, unsigned MAXMASK>
__device__ __forceinline__ void red_init(Red& r) {
#pragma unroll
  for (int k = 0; k < NRED; ++k) r.v[k] = 0.0;
}

template <int NRED, unsigned MAXMASK>
__device__ __forceinline__ void red_combine(Red& a, const Red& b) {
#pragma unroll
  for (int k = 0; k < NRED; ++k) {
    if (MAXMASK & (1u << k)) a.v[k] = nanmax(a.v[k], b.v[k]);
    else a.v[k] = a.v[k] + b.v[k];
  }
}

// Fixed-order warp reduction; lane 0 holds the result.
template <int NRED, unsigned MAXMASK>
__device__ __forceinline__ void warp_reduce(Red& r) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    Red o;
#pragma unroll
    for (int k = 0; k < NRED; ++k) o.v[k] = __shfl_down_sync(0xffffffffu, r.v[k], off);
    if ((threadIdx.x & 31) + off < 32) red_combine<NRED, MAXMASK>(r, o);
  }
}

__device__ __forceinline__ double warp_sum_bcast(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double o = __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) + off < 32) v = v + o;
  }
  return __shfl_sync(0xffffffffu, v, 0);
}

// Fixed-order block reduction for the plain reduction kernels (kThreads
// threads); thread 0 returns the result.
template <int NRED, unsigned MAXMASK>
__device__ void block_reduce(Red& r, double (*s_red)[kThreads / 32]) {
  if constexpr (NRED > 0) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    warp_reduce<NRED, MAXMASK>(r);
    __syncthreads();
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < NRED; ++k) s_red[k][wid] = r.v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
      Red t;
#pragma unroll
      for (int k = 0; k < NRED; ++k) t.v[k] = s_red[k][0];
      for (int w = 1; w < kThreads / 32; ++w) {
        Red o;
#pragma unroll
        for (int k = 0; k < NRED; ++k) o.v[k] = s_red[k][w];
        red_combine<NRED, MAXMASK>(t, o);
      }
      r = t;
    }
    __syncthreads();
  }
}

// Cache operators of the engine's loads (defaults measured best on B200:
// gathers through L2 only, streams and epilogue inputs evict-first):
//   gathers of xin:      0 ld.global.nc, 1 ld.global.cg (L2 only),
//                        2 ld.global.nc.L1::no_allocate, 3 ld.global.cg with
//                          an L2 evict-last policy;
//   col / val streams:   0 ld.global.cs, 1 ld.global.cg,
//                        2 ld.global.nc.L1::no_allocate with an L2 evict-first
//                          policy, 3 ld.global.nc;
//   epilogue inputs:     0 ld.global.cs, 1 ld.global.cg.
#ifndef HPR_ENGINE_GATHER
#define HPR_ENGINE_GATHER 1
#endif
#ifndef HPR_ENGINE_STREAM
#define HPR_ENGINE_STREAM 0
#endif
#ifndef HPR_ENGINE_EPILOAD
#define HPR_ENGINE_EPILOAD 0
#endif

// ---- loads with the cache operators chosen above
__device__ __forceinline__ double ld_nc_na(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_nc_na(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ int32_t ld_stream_pol(const int32_t* p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream_pol(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ double ld_cg_last(const double* p) {
  double v;
  asm("ld.global.cg.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(l2_evict_last_policy()));
  return v;
}
__device__ __forceinline__ float ld_cg_last(const float* p) {
  float v;
  asm("ld.global.cg.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(l2_evict_last_policy()));
  return v;
}
template <class T>
__device__ __forceinline__ T ld_gather(const T* p) {
  if constexpr (HPR_ENGINE_GATHER == 1) return __ldcg(p);
  else if constexpr (HPR_ENGINE_GATHER == 2) return ld_nc_na(p);
  else if constexpr (HPR_ENGINE_GATHER == 3) return ld_cg_last(p);
  else return __ldg(p);
}
template <class T>
__device__ __forceinline__ T ld_stream(const T* p, uint64_t pol) {
  if constexpr (HPR_ENGINE_STREAM == 1) return __ldcg(p);
  else if constexpr (HPR_ENGINE_STREAM == 2) return ld_stream_pol(p, pol);
  else if constexpr (HPR_ENGINE_STREAM == 3) return __ldg(p);
  else return __ldcs(p);
}
template <class T>
__device__ __forceinline__ T ld_epi(const T* p) {
  if constexpr (HPR_ENGINE_EPILOAD == 1) return __ldcg(p);
  else return __ldcs(p);
}

// The epilogue inputs of one row, read by `in(k, i)` like a vector.
template <int NS>
struct Vals {
  double v[NS > 0 ? NS : 1];
  __device__ __forceinline__ double operator()(int k, int64_t) const { return v[k]; }
};

// (the source arrays are selected per slot with compile-time indices so the
// epilogue stays in the kernel-parameter space); the first N slots only
template <class Epi, int N = Epi::kSlots>
__device__ __forceinline__ void load_vals(Vals<Epi::kSlots>& o, const Epi& epi, bool cone, int64_t i) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const double* p = cone ? epi.cone_src[k] : epi.lin_src[k];
    o.v[k] = p ? ld_epi(p + i) : 0.0;
  }
}

// Slots an epilogue's cone_apply reads (Epi::kApplySlots when declared,
// else all of them).
template <class Epi, class = void>
struct ApplySlots {
  static constexpr int value = Epi::kSlots;
};
template <class Epi>
struct ApplySlots<Epi, std::void_t<decltype(Epi::kApplySlots)>> {
  static constexpr int value = Epi::kApplySlots;
};

struct EngineArgs {
  DevCSR M;
  const double* xin;    // gathered vector (FP64 stream)
  const float* xin32;   // gathered vector (reduced-precision streams)
  PlanView pv;
  DevState* st;
  double* red_slots;    // [nslots][kMaxRed] or null
  int bump_inner;       // advance st->inner after the launch
};


// Build-time tuning (defaults measured best on B200): warps per CTA, CTAs
// per SM requested from the register allocator, tiles per atomic grab and
// nonzeros per lane per gather round.
#ifndef HPR_ENGINE_WARPS
#define HPR_ENGINE_WARPS 8
#endif
#ifndef HPR_ENGINE_MINB
#define HPR_ENGINE_MINB 3
#endif
#ifndef HPR_ENGINE_CHUNK
#define HPR_ENGINE_CHUNK 4
#endif
#ifndef HPR_ENGINE_PREFETCH
#define HPR_ENGINE_PREFETCH 0  // 1: epilogue inputs loaded before the gather rounds
#endif
#ifndef HPR_ENGINE_L2PF
#define HPR_ENGINE_L2PF 0  // 1: a tile's column/value stream and epilogue rows are prefetched to L2 at its start;
                           // 2: also the next tile's, after the current tile's gathers (with an early grab)
#endif
#ifndef HPR_ENGINE_EARLYGRAB
#define HPR_ENGINE_EARLYGRAB (HPR_ENGINE_L2PF >= 2)
#endif
#ifndef HPR_ENGINE_PIPE
#define HPR_ENGINE_PIPE 1  // next round's col/val requested before this round's gathers
#endif
#ifndef HPR_ENGINE_PDL
#define HPR_ENGINE_PDL 1  // engine kernels use programmatic dependent launch (0: plain launches)
#endif

constexpr int kWarpsPerCta = HPR_ENGINE_WARPS;
constexpr int kEngineThreads = kWarpsPerCta * 32;
#ifndef HPR_ENGINE_GRAB
#define HPR_ENGINE_GRAB 1
#endif
constexpr int kGrab = HPR_ENGINE_GRAB;  // tiles taken per atomic
constexpr int kChunk = HPR_ENGINE_CHUNK;  // elements per lane per gather round

constexpr bool kTwoRows = kRowCap > 32;   // a lane owns rows lane and lane + 32

// Asynchronous prefetch of a byte range into L2 (no registers, no wait):
// the 16-byte-aligned cover of [p, p + bytes).  Every device array is
// 256-byte aligned with 64 bytes of slack after its end, so the cover stays
// inside the allocation.
__device__ __forceinline__ void prefetch_l2(const void* p, int64_t bytes) {
  if (bytes <= 0) return;
  const uintptr_t b = reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)15;
  const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + (uintptr_t)bytes + 15) & ~(uintptr_t)15;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"((uint32_t)(e - b)) : "memory");
}

struct WarpSmem {
  double acc[kRowCap];  // row sums by non-empty ordinal, then raw cone values by row
  double ns[kRowCap];   // per-cone norms at the cone's first row
  int32_t aux[kRowCap]; // cone heads
};

__device__ __forceinline__ bool tile_is_cone(const Task& t, bool cones) {
  return cones && (t.kind == TASK_CONE_PART || t.cone >= 0);
}

#ifndef HPR_SPIN_LIMIT
#define HPR_SPIN_LIMIT (1 << 22)  // polls of a big cone's ready flag (~0.5 s) before giving up
#endif

__device__ __forceinline__ int ld_acquire(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The last slice of a split cone has arrived: ||tail||_2 from the slices'
// shares (added in slice order), published for the cone's apply tiles.
// Executed by one warp.
inline __device__ void publish_big_norm(const EngineArgs& a, int slot, int nred) {
  const BigCone bc = a.pv.big[slot];
  const int lane = threadIdx.x & 31;
  __threadfence();
  double part = 0.0;
  for (int q = lane; q < bc.nparts; q += 32) part = part + __ldcg(a.pv.cpart + bc.part_base + q);
  const double ns = sqrt(warp_sum_bcast(part));
  if (lane == 0) {
    a.pv.bignorm[slot] = ns;
    // the cone's own reduction slot carries nothing (the apply tiles and the
    // slices carry the rows' terms)
    if (nred > 0)
      for (int k = 0; k < nred; ++k) a.red_slots[(int64_t)(a.pv.ntasks + slot) * kMaxRed + k] = 0.0;
    a.pv.big_cnt[slot] = 0;
    __threadfence();
    atomicExch(a.pv.big_ready + slot, 1);
  }
}

// A slice's share of ||tail||^2: the squares of its raw values, the cone's
// first row excluded, in a fixed order.
__device__ __forceinline__ void big_norm_share(const EngineArgs& a, int slot, int part, double sq) {
  const double tot = warp_sum_bcast(sq);
  if ((threadIdx.x & 31) == 0) a.pv.cpart[a.pv.big[slot].part_base + part] = tot;
}

// Projection of rows [t.rb, t.re) of a split cone (TASK_CONE_APPLY): waits
// for the cone's published norm.  Apply tiles are queued after every slice,
// so the slices were all taken before any apply tile and the wait is short;
// it gives up after HPR_SPIN_LIMIT polls, raising HPR_E_TIMEOUT in the
// device error word, and leaves those rows unprojected.
template <class Epi>
__device__ void cone_apply_task(const EngineArgs& a, Epi& epi, int tix, const Task& t) {
  const int lane = threadIdx.x & 31;
  const int slot = t.group;
  int ok = 1;
  if (lane == 0) {
    int it = 0;
    while (ld_acquire(a.pv.big_ready + slot) == 0) {
      if (++it > HPR_SPIN_LIMIT) {
        ok = 0;
        break;
      }
      __nanosleep(100);
    }
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  Red red;
  red_init<Epi::kNRed, Epi::kMaxMask>(red);
  if (ok) {
    __threadfence();
    const BigCone bc = a.pv.big[slot];
    const double ns = __ldcg(a.pv.bignorm + slot);
    const double tv = __ldcg(a.pv.raw + bc.rb);
    constexpr int kN = ApplySlots<Epi>::value;
    Vals<Epi::kSlots> v0, v1;
    double rv0 = 0.0, rv1 = 0.0;
    const int r0 = t.rb + lane, r1 = t.rb + lane + 32;
    if (r0 < t.re) {
      load_vals<Epi, kN>(v0, epi, true, r0);
      rv0 = __ldcg(a.pv.raw + r0);
    }
    if (kTwoRows && r1 < t.re) {
      load_vals<Epi, kN>(v1, epi, true, r1);
      rv1 = __ldcg(a.pv.raw + r1);
    }
    if (r0 < t.re) epi.cone_apply(r0, rv0, tv, ns, r0 == bc.rb, v0, red);
    if (kTwoRows && r1 < t.re) epi.cone_apply(r1, rv1, tv, ns, r1 == bc.rb, v1, red);
  } else if (lane == 0) {
    atomicExch(&a.st->error, HPR_E_TIMEOUT);
  }
  if constexpr (Epi::kNRed > 0) {
    warp_reduce<Epi::kNRed, Epi::kMaxMask>(red);
    if (lane == 0) {
      double* dst = a.red_slots + (int64_t)tix * kMaxRed;
      for (int k = 0; k < Epi::kNRed; ++k) dst[k] = red.v[k];
    }
  }
  // the cone's last apply tile re-arms its flags for the next launch
  if (lane == 0) {
    const int old = atomicAdd(a.pv.apply_cnt + slot, 1);
    if (old == a.pv.big[slot].napply - 1) {
      a.pv.apply_cnt[slot] = 0;
      a.pv.big_ready[slot] = 0;
    }
  }
}

// Arrival of one slice on a split cone; true (in every lane) for the warp
// that completed it.  Callers must have written their raw values.
__device__ __forceinline__ bool arrive_big(const EngineArgs& a, int slot) {
  __threadfence();  // every lane publishes its raw values
  __syncwarp();
  int last = 0;
  if ((threadIdx.x & 31) == 0) {
    int old = atomicAdd(a.pv.big_cnt + slot, 1);
    last = (old == a.pv.big[slot].nparts - 1) ? 1 : 0;
  }
  return __shfl_sync(0xffffffffu, last, 0) != 0;
}

// Projection and epilogue of a tile's rows once their sums are known (acc0
// for row rb + lane, acc1 for row rb + lane + 32), shared by both layouts.
template <class Epi>
__device__ __forceinline__ void tile_epilogue(const EngineArgs& a, Epi& epi, int tix, const Task& t, bool cone,
                                              int nrows, double acc0, double acc1, const Vals<Epi::kSlots>& v0,
                                              const Vals<Epi::kSlots>& v1, double* ns, WarpSmem& ws, Red& red) {
  const int lane = threadIdx.x & 31;
  if (!cone) {
    if (lane < nrows) epi.linear(t.rb + lane, acc0, v0, red);
    if (kTwoRows && lane + 32 < nrows) epi.linear(t.rb + lane + 32, acc1, v1, red);
    if constexpr (Epi::kNRed > 0) {
      if (t.kind == TASK_CONE_PART && lane == 0) {
        double* dst = a.red_slots + (int64_t)(a.pv.ntasks + t.group) * kMaxRed;
        for (int k = 0; k < Epi::kNRed; ++k) dst[k] = 0.0;
      }
    }
  } else if (t.kind == TASK_CONE_PART) {
    const int head = a.pv.big[t.group].rb;
    double sq = 0.0;
    if (lane < nrows) {
      const double r = epi.cone_raw(t.rb + lane, acc0, v0, red);
      a.pv.raw[t.rb + lane] = r;
      if (t.rb + lane != head) sq = r * r;
    }
    if (kTwoRows && lane + 32 < nrows) {
      const double r = epi.cone_raw(t.rb + lane + 32, acc1, v1, red);
      a.pv.raw[t.rb + lane + 32] = r;
      if (t.rb + lane + 32 != head) sq = sq + r * r;
    }
    big_norm_share(a, t.group, t.part, sq);
    if (arrive_big(a, t.group)) publish_big_norm(a, t.group, Epi::kNRed);
  } else {
    // whole small cones: raw values in place, one lane per cone for the
    // norm (ascending order, like the reference), one lane per row for the
    // projection.
    if (lane < nrows) ws.acc[lane] = epi.cone_raw(t.rb + lane, acc0, v0, red);
    if (kTwoRows && lane + 32 < nrows) ws.acc[lane + 32] = epi.cone_raw(t.rb + lane + 32, acc1, v1, red);
    __syncwarp();
    for (int k = lane; k < t.ncones; k += 32) {
      int c0 = __ldg(a.pv.cone_start + t.cone + k) - t.rb;
      int c1 = __ldg(a.pv.cone_start + t.cone + k + 1) - t.rb;
      double ss = 0.0;
      for (int j = c0 + 1; j < c1; ++j) ss += ws.acc[j] * ws.acc[j];
      ns[c0] = sqrt(ss);
      for (int j = c0; j < c1; ++j) ws.aux[j] = c0;
    }
    __syncwarp();
    if (lane < nrows) {
      int h = ws.aux[lane];
      epi.cone_apply(t.rb + lane, ws.acc[lane], ws.acc[h], ns[h], lane == h, v0, red);
    }
    if (kTwoRows && lane + 32 < nrows) {
      int r = lane + 32, h = ws.aux[r];
      epi.cone_apply(t.rb + r, ws.acc[r], ws.acc[h], ns[h], r == h, v1, red);
    }
  }
  __syncwarp();

  // ---- per-tile reduction slot
  if constexpr (Epi::kNRed > 0) {
    warp_reduce<Epi::kNRed, Epi::kMaxMask>(red);
    if (lane == 0) {
      double* dst = a.red_slots + (int64_t)tix * kMaxRed;
      for (int k = 0; k < Epi::kNRed; ++k) dst[k] = red.v[k];
    }
  }
}

// The last slice of a long row: add the slice partials in slice order and
// finish the row (and its cone, when the row belongs to a split cone).
template <class Epi>
__device__ __forceinline__ void long_row_part(const EngineArgs& a, Epi& epi, int tix, const Task& t, double ps) {
  const int lane = threadIdx.x & 31;
  const LongRow lr = a.pv.lng[t.group];
  int last = 0;
  if (lane == 0) {
    a.pv.partials[lr.partial_base + t.part] = ps;
    __threadfence();
    int old = atomicAdd(a.pv.lng_cnt + t.group, 1);
    last = (old == lr.nparts - 1) ? 1 : 0;
  }
  if (__shfl_sync(0xffffffffu, last, 0)) {
    __threadfence();
    // the lanes load 32 partials at a time and the sum takes them in slice
    // order from the lanes (one L2 round trip per 32 slices)
    double tot = 0.0;
    for (int p0 = 0; p0 < lr.nparts; p0 += 32) {
      const int cnt = min(32, lr.nparts - p0);
      const double mine = lane < cnt ? __ldcg(a.pv.partials + lr.partial_base + p0 + lane) : 0.0;
      for (int j = 0; j < cnt; ++j) tot = tot + __shfl_sync(0xffffffffu, mine, j);
    }
    if (lane == 0) a.pv.lng_cnt[t.group] = 0;
    const bool to_cone = Epi::kCones && lr.bigcone >= 0;
    Red lred;
    red_init<Epi::kNRed, Epi::kMaxMask>(lred);
    if (lane == 0) {
      Vals<Epi::kSlots> v;
      load_vals<Epi>(v, epi, to_cone, lr.row);
      if (!to_cone) {
        epi.linear(lr.row, tot, v, lred);
      } else {
        const double r = epi.cone_raw(lr.row, tot, v, lred);
        a.pv.raw[lr.row] = r;
        // the row's share of its cone's ||tail||^2
        const BigCone bc = a.pv.big[lr.bigcone];
        a.pv.cpart[bc.part_base + lr.cpart] = lr.row == bc.rb ? 0.0 : r * r;
      }
      if constexpr (Epi::kNRed > 0) {
        double* dst = a.red_slots + (int64_t)(a.pv.ntasks + a.pv.nbig + t.group) * kMaxRed;
        for (int k = 0; k < Epi::kNRed; ++k) dst[k] = lred.v[k];
      }
    }
    if (to_cone && arrive_big(a, lr.bigcone)) publish_big_norm(a, lr.bigcone, Epi::kNRed);
  }
  if constexpr (Epi::kNRed > 0) {
    // this tile's own slot carries nothing
    if (lane == 0)
      for (int k = 0; k < Epi::kNRed; ++k) a.red_slots[(int64_t)tix * kMaxRed + k] = 0.0;
  }
}

// L2 prefetch of tile `tix`: its column and value slots (lanes 0, 1) and
// its rows of each epilogue input (lanes 2..), so that the tile's loads after
// the first ones meet L2 instead of DRAM latency.
template <class Epi, int PREC>
__device__ __forceinline__ void prefetch_tile(const EngineArgs& a, const Epi& epi, int tix) {
  const int lane = threadIdx.x & 31;
  if (lane >= 2 + Epi::kSlots) return;
  const Task t = a.pv.tasks[tix];
  if (t.kind == TASK_CONE_APPLY) return;
  if (lane < 2) {
    const int64_t sb = a.pv.runs[tix].sbase;
    const int64_t slots = 32 * (int64_t)((t.nze - t.nzb + 31) >> 5);
    if (lane == 0) prefetch_l2(a.pv.tcol + sb, slots * 4);
    else if constexpr (PREC == HPR_PREC_FP64) prefetch_l2(a.pv.tval + sb, slots * 8);
    else if constexpr (PREC == HPR_PREC_FP32) prefetch_l2(a.pv.tval32 + sb, slots * 4);
    else prefetch_l2(a.pv.tval16 + sb, slots * 2);
    return;
  }
  if (t.kind == TASK_LONG_PART) return;
  // (compile-time slot indices keep the epilogue out of local memory)
  const bool cone = tile_is_cone(t, Epi::kCones);
  const double* src = nullptr;
#pragma unroll
  for (int k = 0; k < Epi::kSlots; ++k)
    if (lane == 2 + k) src = cone ? epi.cone_src[k] : epi.lin_src[k];
  if (src) prefetch_l2(src + t.rb, (int64_t)(t.re - t.rb) * 8);
}

// One tile in the run layout (TileRun).  Lane L owns run L: R = ceil(nnz/32)
// consecutive nonzeros of the tile, stored at slots sbase + 32 k + L.  Per
// step the warp requests U column/value pairs per lane (coalesced, streamed
// evict-first), the next step's pairs, and then the U gathers of xin; each
// lane adds its products in column order (a separate multiply and add, as
// the reference's sequential product), closing a row sum at every row start
// the lane's descriptor marks.  A row inside one run is thus summed exactly
// as the reference sums it.  A row that began in an earlier run (the run's
// first segment) is a continuation: the continuations of one row are added
// in a fixed-order segmented scan over the lanes and then to the row's head
// segment.  Row sums are indexed by non-empty ordinal in shared memory and
// read back by the lanes that own the rows.
// kCoherent: the gathered vector may have been written earlier in the same
// launch (the fused multi-iteration kernel), so it is read through L2
// instead of the read-only path.
// CH (U): nonzeros per lane per step.
// pf_next >= 0: the warp's next tile, prefetched to L2 after this tile's
// gathers.
template <class Epi, int PREC, bool kCoherent = false, int CH = kChunk>
__device__ void process_warp_tile(const EngineArgs& a, Epi& epi, int tix, WarpSmem& ws, int pf_next = -1) {
  constexpr int U = CH;
  const int lane = threadIdx.x & 31;
  const Task* tp = a.pv.tasks + tix;
  if (HPR_ENGINE_L2PF >= 1 && !kCoherent) prefetch_tile<Epi, PREC>(a, epi, tix);
  if (tp->kind == TASK_CONE_APPLY) {
    if constexpr (Epi::kCones) {
      cone_apply_task(a, epi, tix, *tp);
    } else if constexpr (Epi::kNRed > 0) {
      // an epilogue without cones treats cone rows as linear rows: nothing
      // is left to project
      if (lane == 0)
        for (int k = 0; k < Epi::kNRed; ++k) a.red_slots[(int64_t)tix * kMaxRed + k] = 0.0;
    }
    return;
  }
  // only the nonzero range is live during the gathers; the rest of the tile
  // descriptor is read again afterwards (an L1 hit), which keeps registers
  // for nonzeros in flight
  const int nnz = tp->nze - tp->nzb;
  const uint64_t desc = a.pv.desc[(int64_t)tix * 32 + lane];
  const int R = (nnz + 31) >> 5;
  int my = nnz - lane * R;
  my = my < 0 ? 0 : (my > R ? R : my);
  const uint64_t pol = HPR_ENGINE_STREAM == 2 ? l2_evict_first_policy() : 0;
  const uint32_t heads = (uint32_t)desc;
  const int j0 = (int)(desc >> kDescOrdShift);
  Vals<Epi::kSlots> v0, v1;
  if (HPR_ENGINE_PREFETCH && tp->kind != TASK_LONG_PART) {
    const Task t = *tp;
    const bool cone = tile_is_cone(t, Epi::kCones);
    const int nrows = t.re - t.rb;
    if (lane < nrows) load_vals<Epi>(v0, epi, cone, t.rb + lane);
    if (kTwoRows && lane + 32 < nrows) load_vals<Epi>(v1, epi, cone, t.rb + lane + 32);
  }

  // ---- 1. products, added per lane in column order
  const int64_t base = (int64_t)a.pv.runs[tix].sbase + lane;
  double s = 0.0, cont = 0.0;
  int cur = j0 - 1;  // non-empty ordinal of the row being summed
  {
    // one base address per array and step; the U loads of a step sit at
    // fixed offsets from it
    auto load_step = [&](int k0, int32_t* cc, double* vv) {
      const int64_t e0 = base + 32 * (int64_t)k0;
      const int32_t* pc = a.pv.tcol + e0;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u;
        cc[u] = 0;
        vv[u] = 0.0;
        if (k < my) {
          cc[u] = ld_stream(pc + 32 * u, pol);
          if constexpr (PREC == HPR_PREC_FP64) vv[u] = ld_stream(a.pv.tval + e0 + 32 * u, pol);
          else if constexpr (PREC == HPR_PREC_FP32) vv[u] = (double)__ldcs(a.pv.tval32 + e0 + 32 * u);
          else
            vv[u] = (double)__uint_as_float(
                ((unsigned int)__ldcs(reinterpret_cast<const unsigned short*>(a.pv.tval16) + e0 + 32 * u)) << 16);
        }
      }
    };
    int32_t cols[U];
    double vals[U];
    load_step(0, cols, vals);
    for (int k0 = 0; k0 < R; k0 += U) {
      int32_t ncols[U];
      double nvals[U];
      if (HPR_ENGINE_PIPE && k0 + U < R) load_step(k0 + U, ncols, nvals);
      double p[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        p[u] = 0.0;
        if (k0 + u < my) {
          if constexpr (PREC == HPR_PREC_FP64)
            p[u] = vals[u] * (kCoherent ? __ldcg(a.xin + cols[u]) : ld_gather(a.xin + cols[u]));
          else
            p[u] = (double)((float)vals[u] * (kCoherent ? __ldcg(a.xin32 + cols[u]) : ld_gather(a.xin32 + cols[u])));
        }
      }
      if (!HPR_ENGINE_PIPE && k0 + U < R) load_step(k0 + U, ncols, nvals);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u;
        if (k < my) {
          if ((heads >> k) & 1u) {
            // a row starts here: close the previous segment
            if (cur >= j0) ws.acc[cur] = s;
            else cont = s;
            ++cur;
            s = 0.0;
          }
          s = s + p[u];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        cols[u] = ncols[u];
        vals[u] = nvals[u];
      }
    }
  }
  if (my > 0) {
    if (cur >= j0) ws.acc[cur] = s;
    else cont = s;
  }

  if (HPR_ENGINE_L2PF >= 2 && pf_next >= 0) prefetch_tile<Epi, PREC>(a, epi, pf_next);
  const Task t = *tp;
  const int nrows = t.re - t.rb;
  const bool cone = tile_is_cone(t, Epi::kCones);
  Red red;
  red_init<Epi::kNRed, Epi::kMaxMask>(red);
  if (t.kind == TASK_LONG_PART) {
    // ---- partial sum of one long row: the runs in a fixed-order warp sum
    long_row_part(a, epi, tix, t, warp_sum_bcast(cont));
    return;
  }

  // without the prefetch, the epilogue inputs are requested here, so they
  // are not live in registers during the gather steps
  if (!HPR_ENGINE_PREFETCH) {
    if (lane < nrows) load_vals<Epi>(v0, epi, cone, t.rb + lane);
    if (kTwoRows && lane + 32 < nrows) load_vals<Epi>(v1, epi, cone, t.rb + lane + 32);
  }

  // ---- 2. continuations: segmented scan over the lanes, then added to the
  // row's head segment
  {
    const bool has_cont = my > 0 && !(heads & 1u);
    const int key = has_cont ? j0 - 1 : -2 - lane;
    double v = has_cont ? cont : 0.0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, v, d);
      const int ok = __shfl_up_sync(0xffffffffu, key, d);
      if (lane >= d && ok == key) v = o + v;
    }
    const int nk = __shfl_down_sync(0xffffffffu, key, 1);
    __syncwarp();  // head segments are in ws.acc
    if (has_cont && (lane == 31 || nk != key)) ws.acc[key] = ws.acc[key] + v;
    __syncwarp();
  }

  // ---- 3. row sums to the owning lanes (empty rows sum to zero)
  double acc0 = 0.0, acc1 = 0.0;
  {
    const unsigned lt = (1u << lane) - 1u;
    const uint64_t ne = a.pv.runs[tix].nonempty;
    const unsigned b0 = (unsigned)(ne & 0xffffffffull);
    const unsigned b1 = (unsigned)(ne >> 32);
    if ((b0 >> lane) & 1u) acc0 = ws.acc[__popc(b0 & lt)];
    if (kTwoRows && ((b1 >> lane) & 1u)) acc1 = ws.acc[__popc(b0) + __popc(b1 & lt)];
    __syncwarp();
  }

  // ---- 4. epilogue
  tile_epilogue<Epi>(a, epi, tix, t, cone, nrows, acc0, acc1, v0, v1, ws.ns, ws, red);
}

constexpr int kEngineSmem = kWarpsPerCta * (int)sizeof(WarpSmem);

// Shared-memory carveout of an engine kernel, in percent of the 228 KB
// shared-memory maximum: room for exactly the CTAs per SM its register
// budget allows (EngineMinBlocks, with the 1 KB each CTA reserves), so the
// rest of the SM's 256 KB stays L1, where the in-flight gathers and streams
// land.
#ifndef HPR_ENGINE_CARVEOUT
#define HPR_ENGINE_CARVEOUT -1  // >= 0: one fixed carveout for every epilogue
#endif
// room for exactly `ctas` CTAs per SM (with the 1 KB each reserves)
constexpr int engine_carveout(int ctas) { return (ctas * (kEngineSmem + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024); }

// CTAs per SM requested from the register allocator, and nonzeros per lane
// per gather round, per epilogue (an epilogue specialises these where its
// registers call for it).
template <class Epi>
struct EngineMinBlocks {
  static constexpr int value = HPR_ENGINE_MINB;
};
template <class Epi>
struct EngineChunk {
  static constexpr int value = kChunk;
};

// kStatic (host-chosen, only for plans without split cones): first tiles by
// warp index, the rest from the atomic counter counted from nstat, so a
// short launch pays no burst of same-address atomics before its first tile
// (when the static tiles are all the tiles no warp touches the counter),
// and one arrival per CTA on the done counter.  Plans with split cones take
// every tile from the counter: a cone's apply tile waits for its slices,
// and a slice taken from the counter is always on a running warp, while a
// static slice may belong to a CTA that is not resident yet.  (Measured on
// B200: the static form is 3-4% faster on the Q path's short launches and
// 0.5% slower on the benchmark's long ones, so each plan gets its form.)
template <class Epi, int PREC, bool kStatic>
__global__ void __launch_bounds__(kEngineThreads, EngineMinBlocks<Epi>::value) engine_kernel(EngineArgs a, Epi epi) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem* s_ws = reinterpret_cast<WarpSmem*>(smem_raw);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#if HPR_ENGINE_PDL
  // launched as a programmatic dependent: nothing is read before the
  // previous kernel in the stream has completed (a no-op otherwise)
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
  const int ntasks = a.pv.ntasks;
  epi.setup(a.st);
  WarpSmem& ws = s_ws[wid];
  if constexpr (kStatic) {
    const int nstat = a.pv.nbig == 0 ? min(ntasks, (int)gridDim.x * kWarpsPerCta * kGrab) : 0;
    const bool dyn = nstat < ntasks;
    int base = (blockIdx.x * kWarpsPerCta + wid) * kGrab;
    if (base >= nstat) {
      base = ntasks;
      if (dyn && lane == 0) base = nstat + atomicAdd(a.pv.task_ctr, kGrab);
      base = __shfl_sync(0xffffffffu, base, 0);
    }
    while (base < ntasks) {
      for (int q = 0; q < kGrab && base + q < ntasks; ++q)
        process_warp_tile<Epi, PREC, false, EngineChunk<Epi>::value>(a, epi, base + q, ws);
      int next = ntasks;
      if (dyn && lane == 0) next = nstat + atomicAdd(a.pv.task_ctr, kGrab);
      base = __shfl_sync(0xffffffffu, next, 0);
    }
  } else {
    int base = 0;
    if (lane == 0) base = atomicAdd(a.pv.task_ctr, kGrab);
    base = __shfl_sync(0xffffffffu, base, 0);
    while (base < ntasks) {
      // with HPR_ENGINE_EARLYGRAB the next grab is requested before this one
      // is processed, so its atomic latency is hidden behind the tiles
      int next = 0;
      if (HPR_ENGINE_EARLYGRAB && lane == 0) next = atomicAdd(a.pv.task_ctr, kGrab);
      for (int q = 0; q < kGrab && base + q < ntasks; ++q) {
        int pf = -1;
        if (HPR_ENGINE_L2PF >= 2 && HPR_ENGINE_EARLYGRAB && q == kGrab - 1) {
          pf = __shfl_sync(0xffffffffu, next, 0);
          pf = pf < ntasks ? pf : -1;
        }
        process_warp_tile<Epi, PREC, false, EngineChunk<Epi>::value>(a, epi, base + q, ws, pf);
      }
      if (!HPR_ENGINE_EARLYGRAB && lane == 0) next = atomicAdd(a.pv.task_ctr, kGrab);
      base = __shfl_sync(0xffffffffu, next, 0);
    }
  }
#if HPR_ENGINE_PDL
  // no more tiles for this warp: the next kernel may start being scheduled
  asm volatile("griddepcontrol.launch_dependents;");
#endif
  // ---- last arrival: reset the tile counter, advance the Halpern counter
  if constexpr (kStatic) {
    // one arrival per CTA, once all of its warps are past their last grab
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      int tk = atomicAdd(a.pv.done_ctr, 1);
      if (tk == (int)gridDim.x - 1) {
        *a.pv.task_ctr = 0;
        *a.pv.done_ctr = 0;
        if (a.bump_inner) a.st->inner = a.st->inner + 1;
        __threadfence();
      }
    }
  } else {
    if (lane == 0) {
      __threadfence();
      int tk = atomicAdd(a.pv.done_ctr, 1);
      if (tk == (int)(gridDim.x * kWarpsPerCta) - 1) {
        *a.pv.task_ctr = 0;
        *a.pv.done_ctr = 0;
        if (a.bump_inner) a.st->inner = a.st->inner + 1;
        __threadfence();
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Deterministic reductions and maps over plain vectors
// ---------------------------------------------------------------------------
constexpr int kRedGrid = 592;  // 4 CTAs per SM on 148 SMs

// CTAs of a plain reduction over n entries: a fixed function of n (so the
// summation order, and the result, depend on n only), at most kRedGrid, and
// small for small vectors so that concurrent contexts share the device.
inline int red_grid(int64_t n) {
  const int64_t g = (n + 8 * kThreads - 1) / (8 * kThreads);
  return (int)(g < 1 ? 1 : (g > kRedGrid ? kRedGrid : g));
}

template <int NRED, unsigned MASK>
__global__ void __launch_bounds__(kThreads) final_reduce_kernel(const double* __restrict__ slots, int nslots,
                                                                double* __restrict__ out) {
  __shared__ double s_red[kMaxRed][kThreads / 32];
  Red r;
  red_init<NRED, MASK>(r);
  // each thread combines slots threadIdx.x, +kThreads, ... in that order;
  // four slots' loads are issued before they are combined
  int s = threadIdx.x;
  for (; s + 3 * kThreads < nslots; s += 4 * kThreads) {
    Red o[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < NRED; ++k) o[u].v[k] = slots[(int64_t)(s + u * kThreads) * kMaxRed + k];
#pragma unroll
    for (int u = 0; u < 4; ++u) red_combine<NRED, MASK>(r, o[u]);
  }
  for (; s < nslots; s += kThreads) {
    Red o;
#pragma unroll
    for (int k = 0; k < NRED; ++k) o.v[k] = slots[(int64_t)s * kMaxRed + k];
    red_combine<NRED, MASK>(r, o);
  }
  block_reduce<NRED, MASK>(r, s_red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NRED; ++k) out[k] = r.v[k];
}

// First level of a wide slot reduction: CTA b combines the contiguous chunk
// [b * per, (b + 1) * per) of slots in a fixed order (per from nslots and
// the grid size only) into partial slot b.
constexpr int kWideReduceCtas = 148;
template <int NRED, unsigned MASK>
__global__ void __launch_bounds__(kThreads) slot_chunk_kernel(const double* __restrict__ slots, int nslots,
                                                              double* __restrict__ partial) {
  __shared__ double s_red[kMaxRed][kThreads / 32];
  Red r;
  red_init<NRED, MASK>(r);
  const int per = (nslots + gridDim.x - 1) / gridDim.x;
  const int b = blockIdx.x * per, e = b + per < nslots ? b + per : nslots;
  for (int s = b + threadIdx.x; s < e; s += kThreads) {
    Red o;
#pragma unroll
    for (int k = 0; k < NRED; ++k) o.v[k] = slots[(int64_t)s * kMaxRed + k];
    red_combine<NRED, MASK>(r, o);
  }
  block_reduce<NRED, MASK>(r, s_red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NRED; ++k) partial[(int64_t)blockIdx.x * kMaxRed + k] = r.v[k];
}

template <int NRED, unsigned MASK, class F>
__global__ void __launch_bounds__(kThreads) vec_reduce_kernel(int64_t n, F f, double* __restrict__ slots) {
  __shared__ double s_red[kMaxRed][kThreads / 32];
  Red r;
  red_init<NRED, MASK>(r);
  // contiguous chunk per CTA: deterministic for a fixed grid
  int64_t per = (n + gridDim.x - 1) / gridDim.x;
  int64_t b = (int64_t)blockIdx.x * per, e = b + per < n ? b + per : n;
  for (int64_t i = b + threadIdx.x; i < e; i += kThreads) f(i, r);
  block_reduce<NRED, MASK>(r, s_red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NRED; ++k) slots[(int64_t)blockIdx.x * kMaxRed + k] = r.v[k];
}

template <class F>
__global__ void __launch_bounds__(kThreads) vec_map_kernel(int64_t n, F f) {
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) f(i);
}

template <int NRED, unsigned MASK, class F>
inline int vec_reduce(Ctx* c, int64_t n, F f, int red_off) {
  if (n <= 0) {
    HPR_CUDA(c, cudaMemsetAsync(c->d_red_out + red_off, 0, NRED * sizeof(double), c->stream));
    return HPR_OK;
  }
  const int g = red_grid(n);
  vec_reduce_kernel<NRED, MASK, F><<<g, kThreads, 0, c->stream>>>(n, f, c->d_red);
  final_reduce_kernel<NRED, MASK><<<1, kThreads, 0, c->stream>>>(c->d_red, g, c->d_red_out + red_off);
  c->launches += 2;
  HPR_CUDA(c, cudaGetLastError());
  return HPR_OK;
}

template <class F>
inline int vec_map(Ctx* c, int64_t n, F f) {
  if (n <= 0) return HPR_OK;
  int64_t blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  vec_map_kernel<F><<<(int)blocks, kThreads, 0, c->stream>>>(n, f);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  return HPR_OK;
}

// Read back `count` reduction results (and the device error flag).
inline int fetch_red(Ctx* c, int count) {
  HPR_CUDA(c, cudaMemcpyAsync(c->h_red_out, c->d_red_out, count * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  HPR_CUDA(c, cudaMemcpyAsync(&c->h_state->error, &c->d_state->error, sizeof(int32_t), cudaMemcpyDeviceToHost,
                              c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (c->h_state->error != 0)
    return set_err(c, c->h_state->error, "device error flag set");
  return HPR_OK;
}

}  // namespace hpr
