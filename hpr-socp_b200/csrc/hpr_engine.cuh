// hpr_engine.cuh — the fused CSR SpMV + epilogue engine.
//
// One launch computes v = M * xin for every row of a matrix side and hands
// each result to an epilogue functor, so intermediate vectors (A'y, A x_hat,
// z_raw, s_raw) never reach HBM.  Work comes from the host planner
// (hpr_plan.cpp) as cone-aligned tiles:
//
//   1. the tile's nonzeros are streamed with coalesced, evict-first loads of
//      column indices and values; gathered vector entries come through L2;
//      products are staged in shared memory;
//   2. each row is summed from shared memory in ascending column order by one
//      thread (rows of at most kSerialMax nonzeros — bit-identical to the
//      reference's sequential sparse product) or by one warp (longer rows);
//   3. the epilogue runs per row (linear rows / boxed variables) or per cone
//      (one thread per cone computes ||tail||_2 serially, then one thread per
//      row projects), or, for cones larger than one tile, in the CTA that
//      completes the cone's last slice (atomic arrival counter, no waiting);
//   4. optional reductions (sums and NaN-propagating maxima) are combined in a
//      fixed order per CTA and written to one slot per tile, so the final
//      values are independent of scheduling.
//
// The last CTA of a launch may also advance the Halpern counter `inner` (an
// arrival ticket, again with no waiting), which lets a whole iteration run
// from device-resident scalars and be captured in a CUDA graph.
#pragma once

#include "hpr_internal.h"

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

// Fixed-order block reduction; thread 0 returns the result.
template <int NRED, unsigned MAXMASK>
__device__ void block_reduce(Red& r, double (*s_red)[kThreads / 32]) {
  if constexpr (NRED > 0) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      Red o;
#pragma unroll
      for (int k = 0; k < NRED; ++k) o.v[k] = __shfl_down_sync(0xffffffffu, r.v[k], off);
      if (lane + off < 32) red_combine<NRED, MAXMASK>(r, o);
    }
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

// Fixed-order block sum of one value per thread; result broadcast to all.
__device__ __forceinline__ double block_sum_bcast(double v, double* s_tmp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double o = __shfl_down_sync(0xffffffffu, v, off);
    if (lane + off < 32) v = v + o;
  }
  __syncthreads();
  if (lane == 0) s_tmp[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = s_tmp[0];
    for (int w = 1; w < kThreads / 32; ++w) t = t + s_tmp[w];
    s_tmp[kThreads / 32] = t;
  }
  __syncthreads();
  double r = s_tmp[kThreads / 32];
  __syncthreads();
  return r;
}

// Matrix values in the precision of the SpMV stream.
template <int PREC>
struct ValLoad;
template <>
struct ValLoad<HPR_PREC_FP64> {
  __device__ __forceinline__ static double ld(const DevCSR& M, int64_t e) { return __ldcs(M.val + e); }
};
template <>
struct ValLoad<HPR_PREC_FP32> {
  __device__ __forceinline__ static double ld(const DevCSR& M, int64_t e) { return (double)__ldcs(M.val32 + e); }
};
template <>
struct ValLoad<HPR_PREC_BF16> {
  __device__ __forceinline__ static double ld(const DevCSR& M, int64_t e) {
    unsigned short b = __ldcs(reinterpret_cast<const unsigned short*>(M.val16) + e);
    return (double)__uint_as_float(((unsigned int)b) << 16);
  }
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

template <class Epi, int PREC>
__device__ __forceinline__ double gathered_product(const EngineArgs& a, int64_t e, int32_t col) {
  if constexpr (PREC == HPR_PREC_FP64) {
    return ValLoad<PREC>::ld(a.M, e) * __ldg(a.xin + col);
  } else {
    float v = (float)ValLoad<PREC>::ld(a.M, e);
    float xv = __ldg(a.xin32 + col);
    return (double)(v * xv);
  }
}

template <class Epi>
__device__ void finalize_big_cone(const EngineArgs& a, Epi& epi, int slot, double* s_tmp,
                                  double (*s_red)[kThreads / 32]) {
  const BigCone bc = a.pv.big[slot];
  const double* raw = a.pv.raw;
  __threadfence();
  // ||tail||_2 with a fixed-order block reduction
  double part = 0.0;
  for (int r = bc.rb + 1 + threadIdx.x; r < bc.re; r += kThreads) {
    double v = __ldcg(raw + r);
    part = part + v * v;
  }
  double ss = block_sum_bcast(part, s_tmp);
  double ns = sqrt(ss);
  double t = __ldcg(raw + bc.rb);
  Red red;
  red_init<Epi::kNRed, Epi::kMaxMask>(red);
  for (int r = bc.rb + threadIdx.x; r < bc.re; r += kThreads)
    epi.cone_apply(r, __ldcg(raw + r), t, ns, r == bc.rb, red);
  block_reduce<Epi::kNRed, Epi::kMaxMask>(red, s_red);
  if constexpr (Epi::kNRed > 0) {
    if (threadIdx.x == 0) {
      double* dst = a.red_slots + (int64_t)(a.pv.ntasks + slot) * kMaxRed;
      for (int k = 0; k < Epi::kNRed; ++k) dst[k] = red.v[k];
    }
  }
  if (threadIdx.x == 0) a.pv.big_cnt[slot] = 0;
}

// Arrival on a big cone: returns true (in every thread) for the CTA that
// completed it.  Callers must have written their raw values.
__device__ __forceinline__ bool arrive_big(const EngineArgs& a, int slot, int* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    int old = atomicAdd(a.pv.big_cnt + slot, 1);
    *s_flag = (old == a.pv.big[slot].nparts - 1) ? 1 : 0;
  }
  __syncthreads();
  return *s_flag != 0;
}

template <class Epi, int PREC>
__global__ void __launch_bounds__(kThreads) engine_kernel(EngineArgs a, Epi epi) {
  __shared__ double s_prod[kNnzTile];
  __shared__ double s_acc[kRowCap];
  __shared__ int32_t s_rp[kRowCap + 1];
  __shared__ int32_t s_aux[kRowCap];
  __shared__ double s_red[kMaxRed][kThreads / 32];
  __shared__ double s_tmp[kThreads / 32 + 1];
  __shared__ int s_nlong;
  __shared__ int s_flag;

  const Task t = a.pv.tasks[blockIdx.x];
  epi.setup(a.st);
  const int tid = threadIdx.x;
  const int nrows = t.re - t.rb;
  const int nnz = t.nze - t.nzb;
  Red red;
  red_init<Epi::kNRed, Epi::kMaxMask>(red);

  // ---- 1. stage row pointers and products
  if (t.kind != TASK_LONG_PART)
    for (int r = tid; r <= nrows; r += kThreads) s_rp[r] = __ldg(a.M.rowptr + t.rb + r) - t.nzb;
  if (tid == 0) s_nlong = 0;
  {
    constexpr int U = kNnzTile / kThreads;
    int32_t cols[U];
    double prods[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      int e = tid + k * kThreads;
      cols[k] = (e < nnz) ? __ldcs(a.M.col + t.nzb + e) : 0;
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      int e = tid + k * kThreads;
      if (e < nnz) prods[k] = gathered_product<Epi, PREC>(a, (int64_t)t.nzb + e, cols[k]);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      int e = tid + k * kThreads;
      if (e < nnz) s_prod[e] = prods[k];
    }
  }
  __syncthreads();

  if (t.kind == TASK_LONG_PART) {
    // ---- partial sum of one long row
    double part = 0.0;
    for (int e = tid; e < nnz; e += kThreads) part = part + s_prod[e];
    double ps = block_sum_bcast(part, s_tmp);
    const LongRow lr = a.pv.lng[t.group];
    if (tid == 0) {
      a.pv.partials[lr.partial_base + t.part] = ps;
      __threadfence();
      int old = atomicAdd(a.pv.lng_cnt + t.group, 1);
      s_flag = (old == lr.nparts - 1) ? 1 : 0;
    }
    __syncthreads();
    if (s_flag) {
      __threadfence();
      if (tid == 0) {
        double tot = 0.0;
        for (int p = 0; p < lr.nparts; ++p) tot = tot + __ldcg(a.pv.partials + lr.partial_base + p);
        a.pv.lng_cnt[t.group] = 0;
        s_tmp[0] = tot;
      }
      __syncthreads();
      const double tot = s_tmp[0];
      Red lred;
      red_init<Epi::kNRed, Epi::kMaxMask>(lred);
      bool to_cone = Epi::kCones && lr.bigcone >= 0;
      if (!to_cone) {
        if (tid == 0) epi.linear(lr.row, tot, lred);
      } else {
        if (tid == 0) a.pv.raw[lr.row] = epi.cone_raw(lr.row, tot, lred);
      }
      if constexpr (Epi::kNRed > 0) {
        if (tid == 0) {
          double* dst = a.red_slots + (int64_t)(a.pv.ntasks + a.pv.nbig + t.group) * kMaxRed;
          for (int k = 0; k < Epi::kNRed; ++k) dst[k] = lred.v[k];
        }
      }
      if (to_cone) {
        if (arrive_big(a, lr.bigcone, &s_flag)) finalize_big_cone(a, epi, lr.bigcone, s_tmp, s_red);
      } else if constexpr (Epi::kNRed > 0) {
        // a big-cone slot of a non-cone epilogue is written by its parts
      }
    }
  } else {
    // ---- 2. row sums from shared memory
    for (int r = tid; r < nrows; r += kThreads) {
      int b0 = s_rp[r], b1 = s_rp[r + 1];
      if (b1 - b0 <= kSerialMax) {
        double s = 0.0;
        for (int k = b0; k < b1; ++k) s = s + s_prod[k];
        s_acc[r] = s;
      } else {
        int li = atomicAdd(&s_nlong, 1);
        s_aux[li] = r;
      }
    }
    __syncthreads();
    {
      const int lane = tid & 31, wid = tid >> 5;
      for (int li = wid; li < s_nlong; li += kThreads / 32) {
        int r = s_aux[li];
        int b0 = s_rp[r], b1 = s_rp[r + 1];
        double s = 0.0;
        for (int k = b0 + lane; k < b1; k += 32) s = s + s_prod[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, off);
        if (lane == 0) s_acc[r] = s;
      }
    }
    __syncthreads();

    // ---- 3. epilogue
    const bool cones_here = Epi::kCones && (t.kind == TASK_CONE_PART || t.cone >= 0);
    if (!cones_here) {
      for (int r = tid; r < nrows; r += kThreads) epi.linear(t.rb + r, s_acc[r], red);
      if constexpr (Epi::kNRed > 0) {
        if (t.kind == TASK_CONE_PART && tid == 0) {
          double* dst = a.red_slots + (int64_t)(a.pv.ntasks + t.group) * kMaxRed;
          for (int k = 0; k < Epi::kNRed; ++k) dst[k] = 0.0;
        }
      }
    } else if (t.kind == TASK_CONE_PART) {
      for (int r = tid; r < nrows; r += kThreads) a.pv.raw[t.rb + r] = epi.cone_raw(t.rb + r, s_acc[r], red);
      if (arrive_big(a, t.group, &s_flag)) finalize_big_cone(a, epi, t.group, s_tmp, s_red);
    } else {
      // whole small cones: raw values in place, one thread per cone for the
      // norm (ascending order, like the reference), one thread per row for
      // the projection.
      for (int r = tid; r < nrows; r += kThreads) s_acc[r] = epi.cone_raw(t.rb + r, s_acc[r], red);
      __syncthreads();
      double* s_ns = s_prod;  // products are dead; reuse for per-cone norms
      for (int k = tid; k < t.ncones; k += kThreads) {
        int c0 = __ldg(a.pv.cone_start + t.cone + k) - t.rb;
        int c1 = __ldg(a.pv.cone_start + t.cone + k + 1) - t.rb;
        double ss = 0.0;
        for (int j = c0 + 1; j < c1; ++j) ss += s_acc[j] * s_acc[j];
        s_ns[c0] = sqrt(ss);
        for (int j = c0; j < c1; ++j) s_aux[j] = c0;
      }
      __syncthreads();
      for (int r = tid; r < nrows; r += kThreads) {
        int h = s_aux[r];
        epi.cone_apply(t.rb + r, s_acc[r], s_acc[h], s_ns[h], r == h, red);
      }
    }
  }

  // ---- 4. per-tile reduction slot
  if constexpr (Epi::kNRed > 0) {
    block_reduce<Epi::kNRed, Epi::kMaxMask>(red, s_red);
    if (tid == 0) {
      double* dst = a.red_slots + (int64_t)blockIdx.x * kMaxRed;
      for (int k = 0; k < Epi::kNRed; ++k) dst[k] = red.v[k];
    }
  }
  // ---- 5. Halpern counter
  if (a.bump_inner) {
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      int tk = atomicAdd(&a.st->ticket, 1);
      if (tk == (int)gridDim.x - 1) {
        a.st->inner = a.st->inner + 1;
        a.st->ticket = 0;
        __threadfence();
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Deterministic reductions and maps over plain vectors
// ---------------------------------------------------------------------------
constexpr int kRedGrid = 592;  // 4 CTAs per SM on 148 SMs

template <int NRED, unsigned MASK>
__global__ void __launch_bounds__(kThreads) final_reduce_kernel(const double* __restrict__ slots, int nslots,
                                                                double* __restrict__ out) {
  __shared__ double s_red[kMaxRed][kThreads / 32];
  Red r;
  red_init<NRED, MASK>(r);
  for (int s = threadIdx.x; s < nslots; s += kThreads) {
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
  vec_reduce_kernel<NRED, MASK, F><<<kRedGrid, kThreads, 0, c->stream>>>(n, f, c->d_red);
  final_reduce_kernel<NRED, MASK><<<1, kThreads, 0, c->stream>>>(c->d_red, kRedGrid, c->d_red_out + red_off);
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

inline int fetch_red(Ctx* c, int count) {
  HPR_CUDA(c, cudaMemcpyAsync(c->h_red_out, c->d_red_out, count * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

}  // namespace hpr
