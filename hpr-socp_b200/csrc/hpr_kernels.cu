// hpr_kernels.cu — epilogues of the fused engine and their launchers: the HPR
// half-steps, residuals, M-norm, sigma terms, restarts, power iteration and
// unscaling.  Arithmetic follows the reference's operation order (file:line
// beside each epilogue); the library is compiled with -fmad=false so the only
// fused multiply-adds are the explicit fma() calls standing for the
// reference's `muladd`.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>

#include "hpr_epilogues.cuh"

namespace hpr {

// ---------------------------------------------------------------------------
// Small kernels
// ---------------------------------------------------------------------------
__global__ void bump_inner_kernel(DevState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->inner = st->inner + 1;
}

// ---------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------
int upload_plan(Ctx* c, Plan& p) {
  int64_t nt = (int64_t)p.tasks.size();
  HPR_TRY(dev_alloc_n(c, &p.d_tasks, nt));
  HPR_TRY(dev_alloc_n(c, &p.d_big, (int64_t)p.big.size()));
  HPR_TRY(dev_alloc_n(c, &p.d_lng, (int64_t)p.lng.size()));
  HPR_TRY(dev_alloc_n(c, &p.d_big_cnt, (int64_t)p.big.size()));
  HPR_TRY(dev_alloc_n(c, &p.d_lng_cnt, (int64_t)p.lng.size()));
  HPR_TRY(dev_alloc_n(c, &p.d_partials, (int64_t)p.npartials));
  HPR_TRY(dev_alloc_n(c, &p.d_raw, p.nrows));
  HPR_TRY(dev_alloc_n(c, &p.d_ctr, 2));
  if (p.tslots > INT32_MAX)
    return set_err(c, HPR_E_UNSUPPORTED, "matrix too large for the engine's int32 tile layout");
  HPR_TRY(dev_alloc_n(c, &p.d_runs, nt));
  HPR_TRY(dev_alloc_n(c, &p.d_desc, nt * 32));
  const int64_t nb = (int64_t)p.big.size();
  HPR_TRY(dev_alloc_n(c, &p.d_cpart, (int64_t)p.ncparts));
  HPR_TRY(dev_alloc_n(c, &p.d_bignorm, nb));
  HPR_TRY(dev_alloc_n(c, &p.d_big_ready, nb));
  HPR_TRY(dev_alloc_n(c, &p.d_apply_cnt, nb));
  HPR_CUDA(c, cudaMemsetAsync(p.d_big_ready, 0, std::max<int64_t>(1, nb) * sizeof(int32_t), c->stream));
  HPR_CUDA(c, cudaMemsetAsync(p.d_apply_cnt, 0, std::max<int64_t>(1, nb) * sizeof(int32_t), c->stream));
  if (nt) {
    HPR_CUDA(c, cudaMemcpyAsync(p.d_runs, p.runs.data(), nt * sizeof(TileRun), cudaMemcpyHostToDevice, c->stream));
    HPR_CUDA(c, cudaMemcpyAsync(p.d_desc, p.desc.data(), nt * 32 * sizeof(uint64_t), cudaMemcpyHostToDevice,
                                c->stream));
  }
  if (nt)
    HPR_CUDA(c, cudaMemcpyAsync(p.d_tasks, p.tasks.data(), nt * sizeof(Task), cudaMemcpyHostToDevice, c->stream));
  if (!p.big.empty())
    HPR_CUDA(c, cudaMemcpyAsync(p.d_big, p.big.data(), p.big.size() * sizeof(BigCone), cudaMemcpyHostToDevice,
                                c->stream));
  if (!p.lng.empty())
    HPR_CUDA(c, cudaMemcpyAsync(p.d_lng, p.lng.data(), p.lng.size() * sizeof(LongRow), cudaMemcpyHostToDevice,
                                c->stream));
  HPR_CUDA(c, cudaMemsetAsync(p.d_big_cnt, 0, std::max<size_t>(1, p.big.size()) * sizeof(int32_t), c->stream));
  HPR_CUDA(c, cudaMemsetAsync(p.d_lng_cnt, 0, std::max<size_t>(1, p.lng.size()) * sizeof(int32_t), c->stream));
  HPR_CUDA(c, cudaMemsetAsync(p.d_ctr, 0, 2 * sizeof(int32_t), c->stream));
  int64_t need = (int64_t)p.nslots() * kMaxRed;
  if (need > c->red_slots) {
    dev_free(c, c->d_red);
    c->d_red = nullptr;
    c->red_slots = 0;
    HPR_TRY(dev_alloc_n(c, &c->d_red, need));
    c->red_slots = need;
  }
  return HPR_OK;
}

PlanView view_of(const Plan& p, const int32_t* cone_start) {
  PlanView v;
  v.tasks = p.d_tasks;
  v.big = p.d_big;
  v.lng = p.d_lng;
  v.big_cnt = p.d_big_cnt;
  v.lng_cnt = p.d_lng_cnt;
  v.partials = p.d_partials;
  v.raw = p.d_raw;
  v.cone_start = cone_start;
  v.task_ctr = p.d_ctr;
  v.done_ctr = p.d_ctr + 1;
  v.ntasks = (int32_t)p.tasks.size();
  v.nbig = (int32_t)p.big.size();
  v.nlng = (int32_t)p.lng.size();
  v.runs = p.d_runs;
  v.desc = p.d_desc;
  v.cpart = p.d_cpart;
  v.bignorm = p.d_bignorm;
  v.big_ready = p.d_big_ready;
  v.apply_cnt = p.d_apply_cnt;
  v.tcol = p.d_tcol;
  v.tval = p.d_tval;
  v.tval32 = p.d_tval32;
  v.tval16 = p.d_tval16;
  return v;
}

// ---------------------------------------------------------------------------
// Run layout of a matrix (TileRun): one warp per tile copies the tile's
// column indices and values from CSR order to lane-interleaved order; the
// padding slots of the last runs hold column 0 and value 0 (the engine never
// reads them).
// ---------------------------------------------------------------------------
namespace {
template <class T>
__global__ void tile_layout_kernel(const Task* __restrict__ tasks, const TileRun* __restrict__ runs, int ntasks,
                                   const int32_t* __restrict__ col, const T* __restrict__ val,
                                   int32_t* __restrict__ tcol, T* __restrict__ tval) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t ti = w0; ti < ntasks; ti += nw) {
    const Task t = tasks[ti];
    const int32_t nnz = t.nze - t.nzb;
    const int32_t R = (nnz + 31) / 32;
    const int64_t sb = runs[ti].sbase;
    for (int32_t k = 0; k < R; ++k) {
      const int32_t e = lane * R + k;  // element k of this lane's run
      const int64_t d = sb + 32 * (int64_t)k + lane;
      if (e < nnz) {
        if (tcol) tcol[d] = col[t.nzb + e];
        tval[d] = val[t.nzb + e];
      } else {
        if (tcol) tcol[d] = 0;
        tval[d] = T(0.0f);
      }
    }
  }
}

template <class T>
int tile_layout(Ctx* c, const Plan& p, const int32_t* col, const T* val, int32_t* tcol, T* tval) {
  const int nt = (int)p.tasks.size();
  if (nt == 0) return HPR_OK;
  const int blocks = std::min(148 * 8, (nt + 7) / 8);
  tile_layout_kernel<T><<<blocks, 256, 0, c->stream>>>(p.d_tasks, p.d_runs, nt, col, val, tcol, tval);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  return HPR_OK;
}
}  // namespace

int ensure_tiled(Ctx* c, const DevCSR& M, const Plan& p, bool build) {
  if (!build) {
    // allocate only (the first engine use builds the copy)
    const int64_t ns = std::max<int64_t>(p.tslots, 1);
    if (p.tiled_of != (const void*)&M) {
      p.tiled_version = p.tiled_version32 = -1;
      p.tiled_of = &M;
    }
    if (!p.d_tcol) HPR_TRY(dev_alloc_n(c, &p.d_tcol, ns));
    if (!p.d_tval) HPR_TRY(dev_alloc_n(c, &p.d_tval, ns));
    return HPR_OK;
  }
  const bool want32 = M.val32 != nullptr || M.val16 != nullptr;
  const bool ok64 = p.tiled_of == (const void*)&M && p.tiled_version == M.version && p.d_tval;
  const bool ok32 = !want32 || (p.tiled_of == (const void*)&M && p.tiled_version32 == M.version32 &&
                                (!M.val32 || p.d_tval32) && (!M.val16 || p.d_tval16));
  if (ok64 && ok32) return HPR_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HPR_CUDA(c, cudaStreamIsCapturing(c->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone)
    return set_err(c, HPR_E_CUDA, "engine layout must be prepared before a stream capture");
  const int64_t ns = std::max<int64_t>(p.tslots, 1);
  if (p.tiled_of != (const void*)&M) {
    // another matrix of the same plan (Q or F' on planQ): rebuild everything
    p.tiled_version = p.tiled_version32 = -1;
    p.tiled_of = &M;
  }
  if (!ok64) {
    if (!p.d_tcol) HPR_TRY(dev_alloc_n(c, &p.d_tcol, ns));
    if (!p.d_tval) HPR_TRY(dev_alloc_n(c, &p.d_tval, ns));
    HPR_TRY(tile_layout<double>(c, p, M.col, M.val, p.d_tcol, p.d_tval));
    p.tiled_version = M.version;
  }
  if (want32 && (!ok32 || !ok64)) {
    if (M.val32) {
      if (!p.d_tval32) HPR_TRY(dev_alloc_n(c, &p.d_tval32, ns));
      HPR_TRY(tile_layout<float>(c, p, nullptr, M.val32, nullptr, p.d_tval32));
    }
    if (M.val16) {
      if (!p.d_tval16) HPR_TRY(dev_alloc_n(c, &p.d_tval16, ns));
      HPR_TRY(tile_layout<__nv_bfloat16>(c, p, nullptr, M.val16, nullptr, p.d_tval16));
    }
    p.tiled_version32 = M.version32;
  }
  return HPR_OK;
}

int prepare_engine(Ctx* c, bool build) {
  if (!c->uploaded) return HPR_OK;
  HPR_TRY(ensure_tiled(c, c->AT, c->planX, build));
  HPR_TRY(ensure_tiled(c, c->A, c->planY, build));
  if (c->q_kind == HPR_Q_CSR || c->q_kind == HPR_Q_OPERATOR) HPR_TRY(ensure_tiled(c, c->Q, c->planQ, build));
  if (c->q_kind == HPR_Q_DIAG_LOWRANK) {
    HPR_TRY(ensure_tiled(c, c->F, c->planF, build));
    HPR_TRY(ensure_tiled(c, c->FT, c->planQ, build));
  }
  return HPR_OK;
}

namespace {

// Persistent grid size of one engine instantiation (resident CTAs per SM x
// SMs), computed once.
template <class Epi, int PREC, bool kStatic>
int engine_grid(int* smem_bytes) {
  static std::once_flag once;
  static int grid = 1;
  constexpr int dyn = kEngineSmem;
  *smem_bytes = dyn;
  std::call_once(once, [] {
    auto k = engine_kernel<Epi, PREC, kStatic>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    const int carve = HPR_ENGINE_CARVEOUT >= 0 ? (int)(HPR_ENGINE_CARVEOUT)
                                               : engine_carveout(EngineMinBlocks<Epi>::value);
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    int per_sm = 0, dev = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kEngineThreads, dyn);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    grid = std::max(1, per_sm) * std::max(1, sms);
  });
  return grid;
}

// One warp per tile at most: a small problem occupies only the SMs it needs,
// so other streams (other contexts of a serving process) run beside it.
template <class Epi, int PREC, bool kStatic>
void launch_engine_form(Ctx* c, int nt, const EngineArgs& a, const Epi& epi) {
  int dyn = 0;
  const int full = engine_grid<Epi, PREC, kStatic>(&dyn);
  const int g = std::max(1, std::min(full, (nt + kWarpsPerCta - 1) / kWarpsPerCta));
#if HPR_ENGINE_PDL
  // programmatic dependent launch: the kernel may be scheduled while the
  // previous one drains; it waits (griddepcontrol.wait) for that kernel's
  // completion before its first memory access
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)g);
  cfg.blockDim = dim3(kEngineThreads);
  cfg.dynamicSmemBytes = (size_t)dyn;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, engine_kernel<Epi, PREC, kStatic>, a, epi);
#else
  engine_kernel<Epi, PREC, kStatic><<<g, kEngineThreads, dyn, c->stream>>>(a, epi);
#endif
}

// Plans without split cones take their first tiles by warp index
// (engine_kernel's kStatic form); the others take every tile from the
// counter.
template <class Epi, int PREC>
void launch_engine_prec(Ctx* c, int nt, const EngineArgs& a, const Epi& epi) {
  if (a.pv.nbig == 0) launch_engine_form<Epi, PREC, true>(c, nt, a, epi);
  else launch_engine_form<Epi, PREC, false>(c, nt, a, epi);
}

template <class Epi>
int engine_launch(Ctx* c, const DevCSR& M, const Plan& p, const int32_t* cone_start, const double* xin,
                  const float* xin32, const Epi& epi, bool bump, bool with_red, int red_off, bool wide_reduce = false) {
  int nt = (int)p.tasks.size();
  if (nt == 0) {
    if (bump) bump_inner_kernel<<<1, 32, 0, c->stream>>>(c->d_state);
    if (with_red) {
      // no rows: reductions are the identity
      HPR_CUDA(c, cudaMemsetAsync(c->d_red_out + red_off, 0, Epi::kNRed * sizeof(double), c->stream));
    }
    return HPR_OK;
  }
  HPR_TRY(ensure_tiled(c, M, p));
  EngineArgs a;
  a.M = M;
  a.xin = xin;
  a.xin32 = xin32;
  a.pv = view_of(p, cone_start);
  a.st = c->d_state;
  a.red_slots = with_red ? c->d_red : nullptr;
  a.bump_inner = bump ? 1 : 0;
  if (c->precision == HPR_PREC_FP32 && xin32 && M.val32)
    launch_engine_prec<Epi, HPR_PREC_FP32>(c, nt, a, epi);
  else if (c->precision == HPR_PREC_BF16 && xin32 && M.val16)
    launch_engine_prec<Epi, HPR_PREC_BF16>(c, nt, a, epi);
  else
    launch_engine_prec<Epi, HPR_PREC_FP64>(c, nt, a, epi);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  if (with_red) {
    const int ns = p.nslots();
    if (wide_reduce && ns > 2 * kThreads && c->d_red2) {
      // two fixed-order levels: contiguous chunks of slots per CTA, then
      // the chunk sums (one CTA reading tens of thousands of slots is a
      // tenth of a power-iteration step on the benchmark)
      const int g = std::min<int>(kWideReduceCtas, (ns + kThreads - 1) / kThreads);
      slot_chunk_kernel<Epi::kNRed, Epi::kMaxMask><<<g, kThreads, 0, c->stream>>>(c->d_red, ns, c->d_red2);
      final_reduce_kernel<Epi::kNRed, Epi::kMaxMask><<<1, kThreads, 0, c->stream>>>(c->d_red2, g,
                                                                                     c->d_red_out + red_off);
      c->launches += 2;
    } else {
      final_reduce_kernel<Epi::kNRed, Epi::kMaxMask><<<1, kThreads, 0, c->stream>>>(c->d_red, ns,
                                                                                     c->d_red_out + red_off);
      c->launches++;
    }
    HPR_CUDA(c, cudaGetLastError());
  }
  return HPR_OK;
}


// Q v into out (Qmap!, sparse_matrix_operator.jl:27-51); tmp holds F v for
// the diag + F'F operator.
int qmap(Ctx* c, const double* v, double* out, double* tmp) {
  if (c->q_kind == HPR_Q_CSR) {
    return engine_launch(c, c->Q, c->planQ, c->d_var_start, v, nullptr, plain(out), false, false, 0);
  }
  if (c->q_kind == HPR_Q_DIAG_LOWRANK) {
    HPR_TRY(engine_launch(c, c->F, c->planF, nullptr, v, nullptr, plain(tmp), false, false, 0));
    return engine_launch(c, c->FT, c->planQ, c->d_var_start, tmp, nullptr, plain(out, c->qdiag, v), false, false,
                         0);
  }
  if (c->q_kind == HPR_Q_OPERATOR) {
    // the caller's Q v, enqueued on the context stream (Qmap! of a user
    // AbstractQOperator)
    c->q_fn(c->q_user, v, out, c->n, (void*)c->stream);
    c->launches++;
    HPR_CUDA(c, cudaGetLastError());
    return HPR_OK;
  }
  HPR_CUDA(c, cudaMemsetAsync(out, 0, c->n * sizeof(double), c->stream));
  return HPR_OK;
}

struct DotF {
  const double *a, *b;
  __device__ void operator()(int64_t i, Red& r) const { r.v[0] = r.v[0] + a[i] * b[i]; }
};
struct Dot2F {
  const double *a, *b, *c, *d;
  __device__ void operator()(int64_t i, Red& r) const {
    r.v[0] = r.v[0] + a[i] * b[i];
    r.v[1] = r.v[1] + c[i] * d[i];
  }
};
struct AbsMaxF {
  const double* a;
  __device__ void operator()(int64_t i, Red& r) const { r.v[0] = nanmax(r.v[0], fabs(a[i])); }
};

}  // namespace

// ---------------------------------------------------------------------------
// Iteration
// ---------------------------------------------------------------------------
int push_state(Ctx* c) {
  c->h_state->sigma = c->sigma;
  c->h_state->lamA = c->lamA;
  c->h_state->lamQ = c->lamQ;
  c->h_state->pad0 = 0;
  c->h_state->inner = c->inner;
  c->h_state->ticket = 0;
  c->h_state->error = 0;
  HPR_CUDA(c, cudaMemcpyAsync(c->d_state, c->h_state, sizeof(DevState), cudaMemcpyHostToDevice, c->stream));
  // the staging buffer is reused: make the copy complete before returning
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

int update_q_factors(Ctx* c) {
  // unified_update_Q_factors! (unified_operations.jl:484-498)
  if (!c->Q_is_diag || !c->has_q) return HPR_OK;
  double s = c->sigma, s2 = s * s;
  const double* dq = c->diag_Q;
  double *f2 = c->fact2, *f = c->fact, *f1 = c->fact1, *fm = c->fact_M;
  return vec_map(c, c->n, [=] __device__(int64_t i) {
    double t2 = 1.0 / (1.0 + s * dq[i]);
    f2[i] = t2;
    f[i] = s * t2;
    f1[i] = s * dq[i] * t2;
    fm[i] = s2 * t2;
  });
}

namespace {

}  // namespace

int launch_iteration(Ctx* c, bool full) {
  const bool fp32 = c->precision != HPR_PREC_FP64;
  IterEpis E;
  make_iter_epis(c, full, E);
  if (!c->has_q) {
    // main_update_noQ_soc_gpu! (algorithm.jl:2302-2309)
    HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->y, fp32 ? c->g32_m : nullptr, E.ex, c->m == 0,
                          false, 0));
    if (c->m > 0)
      HPR_TRY(engine_launch(c, c->A, c->planY, c->d_con_start, c->x_hat, fp32 ? c->g32_n : nullptr, E.ey, true, false,
                            0));
    return HPR_OK;
  }
  // Q path: zxw1, y, w2 (algorithm.jl:2291-2295)
  const bool lowrank = c->q_kind == HPR_Q_DIAG_LOWRANK;
  if (lowrank) {
    HPR_TRY(engine_launch(c, c->F, c->planF, nullptr, c->w, nullptr, plain(c->ftmp), false, false, 0));
    HPR_TRY(engine_launch(c, c->FT, c->planQ, c->d_var_start, c->ftmp, nullptr, E.eq, false, false, 0));
  } else if (c->q_kind == HPR_Q_OPERATOR) {
    // Q w from the caller's operator; the epilogue runs over the identity
    HPR_TRY(qmap(c, c->w, c->qop_out, nullptr));
    HPR_TRY(engine_launch(c, c->Q, c->planQ, c->d_var_start, c->qop_out, nullptr, E.eq, false, false, 0));
  } else {
    HPR_TRY(engine_launch(c, c->Q, c->planQ, c->d_var_start, c->w, nullptr, E.eq, false, false, 0));
  }
  if (c->m > 0) {
    if (lowrank) {
      HPR_TRY(engine_launch(c, c->F, c->planF, nullptr, c->w_bar, nullptr, plain(c->ftmp2), false, false, 0));
      HPR_TRY(engine_launch(c, c->FT, c->planQ, c->d_var_start, c->ftmp2, nullptr, E.et, false, false, 0));
    } else if (c->q_kind == HPR_Q_OPERATOR) {
      HPR_TRY(qmap(c, c->w_bar, c->qop_out, nullptr));
      HPR_TRY(engine_launch(c, c->Q, c->planQ, c->d_var_start, c->qop_out, nullptr, E.et, false, false, 0));
    } else {
      HPR_TRY(engine_launch(c, c->Q, c->planQ, c->d_var_start, c->w_bar, nullptr, E.et, false, false, 0));
    }
    HPR_TRY(engine_launch(c, c->A, c->planY, c->d_con_start, c->tempv, fp32 ? c->g32_n : nullptr, E.ey, false, false,
                          0));
  }
  return engine_launch(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, E.e2, true, false, 0);
}

// ---------------------------------------------------------------------------
// Fused multi-iteration kernel for small problems.
//
// When every matrix side fits a few tiles per warp, one CTA runs k whole
// iterations in a single launch: its warps split each half-step's tiles
// statically, a CTA barrier separates the half-steps (the next half-step
// gathers what the previous one wrote, through L2), and thread 0 advances
// the Halpern counter after each iteration.  This replaces 2-4 launches per
// iteration by one launch per batch, which is what bounds small solves and
// lets many of them share the device.  Arithmetic and order per row are
// those of the engine, so results are identical to the unfused path.
// ---------------------------------------------------------------------------

namespace {

// Stages run in order each iteration; `full_last` selects the full
// epilogues on the last iteration.
template <class E0, class E1, class E2, class E3, int PREC>
__global__ void __launch_bounds__(kEngineThreads, 1)
    fused_kernel(FStage<E0> s0, FStage<E1> s1, FStage<E2> s2, FStage<E3> s3, DevState* st, int iters, int full_last) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(smem_raw)[threadIdx.x >> 5];
  for (int it = 0; it < iters; ++it) {
    const bool last = full_last && it + 1 == iters;
    fused_stage<E0, PREC>(s0, last, ws);
    fused_stage<E1, PREC>(s1, last, ws);
    fused_stage<E2, PREC>(s2, last, ws);
    fused_stage<E3, PREC>(s3, last, ws);
    if (threadIdx.x == 0) st->inner = st->inner + 1;
    __syncthreads();
  }
}

// The single-CTA kernels use the engine's per-warp buffers (kEngineSmem);
// above 48 KB a kernel needs the opt-in attribute, set once per kernel.
constexpr int kSmemOptinMax = 227 * 1024;
template <class K>
int allow_engine_smem(Ctx* c, K kernel) {
  if (kEngineSmem <= 48 * 1024) return HPR_OK;
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;  // (device, kernel)
  const std::pair<int, const void*> key(c->device, (const void*)kernel);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(key)) return HPR_OK;
  HPR_CUDA(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kEngineSmem));
  done.insert(key);
  return HPR_OK;
}

template <class E0, class E1, class E2, class E3>
int launch_fused_prec(Ctx* c, const FStage<E0>& s0, const FStage<E1>& s1, const FStage<E2>& s2, const FStage<E3>& s3,
                      int iters, int full_last) {
  const int prec = c->precision;
  auto go = [&](auto kernel) {
    HPR_TRY(allow_engine_smem(c, kernel));
    kernel<<<1, kEngineThreads, kEngineSmem, c->stream>>>(s0, s1, s2, s3, c->d_state, iters, full_last);
    return HPR_OK;
  };
  if (prec == HPR_PREC_FP32 && s0.a.M.val32) HPR_TRY(go(fused_kernel<E0, E1, E2, E3, HPR_PREC_FP32>));
  else if (prec == HPR_PREC_BF16 && s0.a.M.val16) HPR_TRY(go(fused_kernel<E0, E1, E2, E3, HPR_PREC_BF16>));
  else HPR_TRY(go(fused_kernel<E0, E1, E2, E3, HPR_PREC_FP64>));
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  return HPR_OK;
}

bool fused_eligible(const Ctx* c) {
  if (c->q_kind == HPR_Q_DIAG_LOWRANK || c->q_kind == HPR_Q_OPERATOR) return false;
  auto fits = [](const Plan& p) { return (int64_t)p.tasks.size() <= kFusedMaxTiles; };
  if (!fits(c->planX) || !fits(c->planY)) return false;
  // with Q the reduced-precision streams apply to A only; keep those unfused
  if (c->has_q && (!fits(c->planQ) || c->precision != HPR_PREC_FP64)) return false;
  return kEngineSmem <= kSmemOptinMax;
}

// k iterations (the last one full when full_last) in one launch.
int launch_fused(Ctx* c, int64_t k, bool full_last) {
  HPR_TRY(prepare_engine(c));
  const bool fp32 = c->precision != HPR_PREC_FP64;
  IterEpis P, F;
  make_iter_epis(c, false, P);
  make_iter_epis(c, true, F);
  const bool hy = c->m > 0;
  for (int64_t done = 0; done < k;) {
    const int n = (int)std::min<int64_t>(k - done, 1 << 20);
    const int fl = (full_last && done + n == k) ? 1 : 0;
    if (!c->has_q) {
      auto sx = fstage(c, c->AT, c->planX, c->d_var_start, c->y, fp32 ? c->g32_m : nullptr, P.ex, F.ex, true);
      auto sy = fstage(c, c->A, c->planY, c->d_con_start, c->x_hat, fp32 ? c->g32_n : nullptr, P.ey, F.ey, hy);
      auto off = fstage(c, c->A, c->planY, c->d_con_start, c->x_hat, nullptr, P.ey, F.ey, false);
      HPR_TRY(launch_fused_prec(c, sx, sy, off, off, n, fl));
    } else {
      auto sq = fstage(c, c->Q, c->planQ, c->d_var_start, c->w, nullptr, P.eq, F.eq, true);
      auto st = fstage(c, c->Q, c->planQ, c->d_var_start, c->w_bar, nullptr, P.et, F.et, hy);
      auto sy = fstage(c, c->A, c->planY, c->d_con_start, c->tempv, fp32 ? c->g32_n : nullptr, P.ey, F.ey, hy);
      auto sw = fstage(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, P.e2, F.e2, true);
      HPR_TRY(launch_fused_prec(c, sq, st, sy, sw, n, fl));
    }
    done += n;
  }
  return HPR_OK;
}

}  // namespace



namespace {

// Unfused path: engine launches (graph replays where captured).
int run_engine_iterations(Ctx* c, int64_t k, bool full_last) {
  int64_t partial = full_last ? k - 1 : k;
  int64_t done = 0;
  // replay the captured partial-iteration graph where it fits
  if (c->graph_partial && c->graph_iters > 0) {
    while (partial - done >= c->graph_iters) {
      HPR_CUDA(c, cudaGraphLaunch(c->graph_partial, c->stream));
      done += c->graph_iters;
      c->launches += c->graph_iters * (c->has_q ? 4 : 2);
    }
  }
  for (; done < partial; ++done) HPR_TRY(launch_iteration(c, false));
  if (full_last) HPR_TRY(launch_iteration(c, true));
  return HPR_OK;
}

// Schedule autotuner.  Problems small enough for the single-CTA fused kernel
// can also run on the multi-CTA engine; which is faster depends on how many
// tiles a side has.  The first batch of at least 16 iterations of a size
// class runs half on each path (the iterates are identical either way),
// times both with events and records the faster per iteration for the
// class; later batches of the class in this process use the recorded choice.
std::mutex g_tune_mu;
std::map<int, int> g_tune;  // class -> HPR_SCHEDULE_ENGINE / _FUSED

int tune_class(const Ctx* c) {
  int64_t t = std::max<int64_t>((int64_t)c->planX.tasks.size(), (int64_t)c->planY.tasks.size());
  if (c->has_q) t = std::max<int64_t>(t, (int64_t)c->planQ.tasks.size());
  int b = 0;
  while ((1LL << b) < t) ++b;
  return (c->has_q ? 100 : 0) + b;
}

int tune_lookup(const Ctx* c) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_class(c));
  return it == g_tune.end() ? HPR_SCHEDULE_AUTO : it->second;
}

int tune_trial(Ctx* c, int64_t k, bool full_last) {
  if (!c->ev_mid) HPR_CUDA(c, cudaEventCreate(&c->ev_mid));
  const int64_t k1 = k / 2;
  HPR_TRY(launch_fused(c, k1, false));
  HPR_CUDA(c, cudaEventRecord(c->ev_mid, c->stream));
  HPR_TRY(run_engine_iterations(c, k - k1, full_last));
  HPR_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  HPR_CUDA(c, cudaEventSynchronize(c->ev1));
  float tf = 0.f, te = 0.f;
  HPR_CUDA(c, cudaEventElapsedTime(&tf, c->ev0, c->ev_mid));
  HPR_CUDA(c, cudaEventElapsedTime(&te, c->ev_mid, c->ev1));
  const int pick = (tf / (double)k1 <= te / (double)(k - k1)) ? HPR_SCHEDULE_FUSED : HPR_SCHEDULE_ENGINE;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.emplace(tune_class(c), pick);
  return HPR_OK;
}

}  // namespace

bool uses_fused_iterations(const Ctx* c) {
  if (!fused_eligible(c)) return false;
  const int mode = c->schedule != HPR_SCHEDULE_AUTO ? c->schedule : tune_lookup(c);
  return mode != HPR_SCHEDULE_ENGINE;
}

int run_iterations(Ctx* c, int64_t k, bool full_last) {
  if (k <= 0) return HPR_OK;
  int64_t l0 = c->launches;
  HPR_CUDA(c, cudaEventRecord(c->ev0, c->stream));
  int mode = HPR_SCHEDULE_ENGINE;
  if (fused_eligible(c)) {
    mode = c->schedule != HPR_SCHEDULE_AUTO ? c->schedule : tune_lookup(c);
    if (mode == HPR_SCHEDULE_AUTO) {
      if (k >= 16) {
        HPR_TRY(tune_trial(c, k, full_last));
        c->inner += k;
        c->last_launches = c->launches - l0;
        return HPR_OK;
      }
      mode = HPR_SCHEDULE_FUSED;
    }
  }
  if (mode == HPR_SCHEDULE_FUSED) HPR_TRY(launch_fused(c, k, full_last));
  else HPR_TRY(run_engine_iterations(c, k, full_last));
  HPR_CUDA(c, cudaEventRecord(c->ev1, c->stream));
  c->inner += k;
  c->last_launches = c->launches - l0;
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// Residuals (compute_residuals!, algorithm.jl:113-196)
// ---------------------------------------------------------------------------
namespace {
__global__ void bounds_box_kernel(int64_t n, const double* l, const double* u, const double* xb, const double* col,
                                  double bs, double* dx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double lv = cmax(l[i] - xb[i], 0.0);
    double uv = cmax(xb[i] - u[i], 0.0);
    dx[i] = (lv + uv) * (bs / col[i]);
  }
}
// compute_err_soc_kernel! (kernels.jl:6617-6655)
__global__ void bounds_cone_kernel(int64_t ncones, const int32_t* vs, const double* xb, const double* col, double bs,
                                   double* dx) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ncones; k += (int64_t)gridDim.x * blockDim.x) {
    int64_t st = vs[k], en = vs[k + 1];
    double t = xb[st];
    double ns = 0.0;
    dx[st] = t;
    for (int64_t j = st + 1; j < en; ++j) {
      dx[j] = xb[j];
      ns += xb[j] * xb[j];
    }
    ns = sqrt(ns);
    if (ns <= -t) {
    } else if (ns <= t) {
      for (int64_t j = st; j < en; ++j) dx[j] = 0.0;
    } else {
      double f = (1 + t / ns) / 2;
      dx[st] = (ns + t) / 2 - t;
      for (int64_t j = st + 1; j < en; ++j) dx[j] = f * dx[j] - dx[j];
    }
    for (int64_t j = st; j < en; ++j) dx[j] *= bs / col[j];
  }
}
}  // namespace

int launch_residuals(Ctx* c, bool include_bounds, hpr_residuals* r) {
  const double bs = c->b_scale, cs = c->c_scale;
  const bool skipq = !c->has_q;
  // offsets in d_red_out: [0..5] Rd lanes, [8..12] Rp lanes, [16] bounds
  if (!skipq) HPR_TRY(qmap(c, c->x_bar, c->Qx, c->ftmp));
  EpiRd ed{};
  const double* dsrc[5] = {c->c, c->z_bar, c->x_bar, c->col_norm, skipq ? nullptr : c->Qx};
  for (int k = 0; k < 5; ++k) ed.lin_src[k] = ed.cone_src[k] = dsrc[k];
  ed.hasq = skipq ? 0 : 1;
  ed.cs = cs;
  HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, ed, false, true, 0));
  if (c->m > 0) {
    EpiRp ep{};
    const double* psrc[5] = {c->AL, c->AU, c->row_norm, c->y_bar, c->s};
    const double* pcone[5] = {c->soc_rhs_full, nullptr, c->row_norm, c->y_bar, c->s};
    for (int k = 0; k < 5; ++k) {
      ep.lin_src[k] = psrc[k];
      ep.cone_src[k] = pcone[k];
    }
    ep.bs = bs;
    HPR_TRY(engine_launch(c, c->A, c->planY, c->d_con_start, c->x_bar, nullptr, ep, false, true, 8));
  }
  if (include_bounds) {
    bounds_box_kernel<<<592, kThreads, 0, c->stream>>>(c->n, c->l, c->u, c->x_bar, c->col_norm, bs, c->dx);
    int64_t nv = (int64_t)c->h_var_idx.size() - 1;
    if (nv > 0)
      bounds_cone_kernel<<<(int)std::min<int64_t>((nv + 127) / 128, 1184), 128, 0, c->stream>>>(
          nv, c->d_var_start, c->x_bar, c->col_norm, bs, c->dx);
    HPR_CUDA(c, cudaGetLastError());
    HPR_TRY(vec_reduce<1, 1>(c, c->n, AbsMaxF{c->dx}, 16));
  }
  HPR_TRY(fetch_red(c, 17));
  const double* h = c->h_red_out;
  auto jmax = [](double a, double b) { return (a != a) ? a : ((b != b) ? b : (a > b ? a : b)); };
  double qx_dot = skipq ? 0.0 : h[5];
  r->primal_obj_bar = bs * cs * (h[3] + 0.5 * qx_dot) + c->obj_constant;
  r->dual_obj_bar = bs * cs * (-0.5 * qx_dot + h[4]) + c->obj_constant;
  if (c->m > 0) r->dual_obj_bar += bs * cs * (h[11] + h[12]);
  r->rel_gap_bar = std::fabs(r->primal_obj_bar - r->dual_obj_bar) /
                   (1.0 + std::max(std::fabs(r->primal_obj_bar), std::fabs(r->dual_obj_bar)));
  double qx_inf = skipq ? 0.0 : h[2];
  r->err_Rd_org_bar = h[0] / (1.0 + jmax(jmax(c->norm_c_org, h[1]), qx_inf));
  if (c->m > 0) {
    double denom = 1.0 + jmax(c->norm_b_org, h[10]);
    double lin = c->m_lin > 0 ? h[8] / denom : 0.0;
    double soc = c->m_lin < c->m ? h[9] / denom : 0.0;
    r->err_Rp_linear_org_bar = lin;
    r->err_Rp_soc_org_bar = soc;
    r->err_Rp_org_bar = jmax(h[8], h[9]) / denom;
  } else {
    r->err_Rp_org_bar = r->err_Rp_linear_org_bar = r->err_Rp_soc_org_bar = 0.0;
  }
  if (include_bounds) r->err_Rp_org_bar = jmax(r->err_Rp_org_bar, h[16]);
  r->KKTx_and_gap_org_bar = jmax(jmax(r->err_Rp_org_bar, r->err_Rd_org_bar), r->rel_gap_bar);
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// M-norm (compute_M_norm!, algorithm.jl:1302-1359)
// ---------------------------------------------------------------------------
int launch_mnorm(Ctx* c, double* out) {
  const double sg = c->sigma;
  const bool skipq = !c->has_q;
  // [0] dx'dx, [1] dy'dy, [2] <A'dy, dx>, [3] dQw'dx, [4] dQw'ATdy,
  // [5] ATdy'QATdy (diag: scaled by fact_M), [6] dQw'dQw, [7] dw'dQw
  double h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  HPR_TRY(vec_reduce<1, 0>(c, c->n, DotF{c->dx, c->dx}, 0));
  if (c->m > 0) HPR_TRY(vec_reduce<1, 0>(c, c->m, DotF{c->dy, c->dy}, 1));
  if (!skipq) {
    HPR_TRY(qmap(c, c->dw, c->dQw, c->ftmp));
    HPR_TRY(vec_reduce<2, 0>(c, c->n, Dot2F{c->dQw, c->dx, c->dQw, c->dQw}, 3));  // [3], [4]=dQw'dQw tmp
  }
  if (c->m > 0) {
    EpiDot e{};
    e.lin_src[0] = e.cone_src[0] = c->dx;
    e.out = c->ATdy;
    HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->dy, nullptr, e, false, true, 2));
  }
  HPR_TRY(fetch_red(c, 8));
  for (int k = 0; k < 5; ++k) h[k] = c->h_red_out[k];
  double dqw2 = h[4];
  double M1 = 0.0, M2 = (1.0 / sg) * h[0], M3 = 0.0;
  if (!skipq) M2 -= 2.0 * h[3];
  if (c->m > 0) {
    M1 = sg * c->lamA * h[1];
    if (!skipq) {
      HPR_TRY(qmap(c, c->ATdy, c->QATdy, c->ftmp));
      const double* fm = c->fact_M;
      double* atdy = c->ATdy;
      bool dg = c->Q_is_diag;
      HPR_TRY(vec_reduce<1, 0>(c, c->n, DotF{c->dQw, c->ATdy}, 0));
      HPR_TRY(fetch_red(c, 1));
      M1 -= 2.0 * sg * c->h_red_out[0];
      M2 += 2.0 * h[2];
      if (dg) HPR_TRY(vec_map(c, c->n, [=] __device__(int64_t i) { atdy[i] *= fm[i]; }));
      HPR_TRY(vec_reduce<2, 0>(c, c->n, Dot2F{c->ATdy, c->QATdy, c->dw, c->dQw}, 0));
      HPR_TRY(fetch_red(c, 2));
      if (dg) {
        M3 = c->h_red_out[0];
        M1 += sg * dqw2;
      } else {
        M3 = (sg * sg) / (1.0 + sg * c->lamQ) * c->h_red_out[0];
        M1 += sg * c->lamQ * c->h_red_out[1];
      }
    } else {
      M2 += 2.0 * h[2];
    }
  } else if (!c->Q_is_diag && !skipq) {
    HPR_TRY(vec_reduce<1, 0>(c, c->n, DotF{c->dw, c->dQw}, 0));
    HPR_TRY(fetch_red(c, 1));
    M1 = sg * c->lamQ * c->h_red_out[0];
  }
  M2 += std::max(M1, 0.0);
  double M = std::max(M2, 0.0) + std::max(M3, 0.0);
  *out = std::sqrt(M);
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// update_sigma! inner products (algorithm.jl:787-833)
// ---------------------------------------------------------------------------
namespace {
struct DiffDotF {
  const double *a, *b;
  double* d;
  __device__ void operator()(int64_t i, Red& r) const {
    double v = a[i] - b[i];
    d[i] = v;
    r.v[0] = r.v[0] + v * v;
  }
};
}  // namespace

int launch_sigma_terms(Ctx* c, double* a, double* b, double* cc, double* d) {
  const bool skipq = !c->has_q;
  const int64_t n = c->n, m = c->m;
  if (!skipq) {
    const double *wb = c->w_bar, *lw = c->last_w;
    double* dw = c->dw;
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { dw[i] = wb[i] - lw[i]; }));
    HPR_TRY(qmap(c, c->dw, c->dQw, c->ftmp));
  }
  HPR_TRY(vec_reduce<1, 0>(c, n, DiffDotF{c->x_bar, c->last_x, c->dx}, 0));
  if (m > 0) HPR_TRY(vec_reduce<1, 0>(c, m, DiffDotF{c->y_bar, c->last_y, c->dy}, 1));
  if (!skipq && m > 0) {
    HPR_TRY(vec_reduce<1, 0>(c, n, DiffDotF{c->ATy_bar, c->last_ATy, c->ATdy}, 7));
    HPR_TRY(qmap(c, c->ATdy, c->QATdy, c->ftmp));
    HPR_TRY(vec_reduce<2, 0>(c, n, Dot2F{c->dQw, c->ATdy, c->ATdy, c->QATdy}, 2));
  }
  if (!skipq) HPR_TRY(vec_reduce<2, 0>(c, n, Dot2F{c->dQw, c->dQw, c->dw, c->dQw}, 4));
  HPR_TRY(fetch_red(c, 8));
  const double* h = c->h_red_out;
  double A = 0.0, B = h[0], C = 0.0, D = 0.0;
  if (m > 0) {
    if (!skipq) A = c->lamA * h[1] - 2.0 * h[2];
    else A = c->lamA * h[1];
  }
  if (!skipq) {
    if (c->Q_is_diag) {
      double nq = std::sqrt(h[4]);
      A += nq * nq;
    } else {
      A += c->lamQ * h[5];
      if (m > 0) {
        C = h[3];
        D = c->lamQ;
      }
    }
  }
  *a = A;
  *b = B;
  *cc = C;
  *d = D;
  return HPR_OK;
}

// unified_golden_Q_diag (unified_operations.jl:411-449): each evaluation is
// one fused pass over diag(Q), A'dy and Q A'dy.
namespace {
// vectors up to this length run the golden-section search in one CTA
#ifndef HPR_GOLDEN_DEVICE_MAX_N
#define HPR_GOLDEN_DEVICE_MAX_N 65536
#endif
constexpr int64_t kGoldenDeviceMaxN = HPR_GOLDEN_DEVICE_MAX_N;
struct GoldenF {
  const double *dq, *c, *d;
  double x;
  __device__ void operator()(int64_t i, Red& r) const { r.v[0] = r.v[0] + c[i] * (d[i] / (1.0 + x * dq[i])); }
};
}  // namespace

namespace {
// The whole golden-section search of unified_golden_Q_diag in one CTA, for
// vectors short enough that one CTA reduces them quickly: each evaluation
// sums the terms in the order of the host-driven search below (chunk j of
// red_grid(n) as vec_reduce_kernel's CTA j, then the chunk sums as
// final_reduce_kernel), and thread 0 runs the same interval updates, so the
// result is the same to the bit without a host round trip per evaluation.
__global__ void __launch_bounds__(kThreads)
    golden_diag_kernel(int64_t n, int g, const double* __restrict__ dq, const double* __restrict__ cv,
                       const double* __restrict__ dv, double a, double b, double lo, double hi, double tol,
                       int maxiter, double* __restrict__ out) {
  __shared__ double s_red[kMaxRed][kThreads / 32];
  __shared__ double s_slot[kRedGrid];
  __shared__ double s_f;
  __shared__ int s_go;
  auto eval = [&](double x) {
    const int64_t per = (n + g - 1) / g;
    for (int j = 0; j < g; ++j) {
      Red r;
      red_init<1, 0>(r);
      const int64_t bb = (int64_t)j * per, ee = bb + per < n ? bb + per : n;
      for (int64_t i = bb + threadIdx.x; i < ee; i += kThreads) r.v[0] = r.v[0] + cv[i] * (dv[i] / (1.0 + x * dq[i]));
      block_reduce<1, 0>(r, s_red);
      if (threadIdx.x == 0) s_slot[j] = r.v[0];
    }
    __syncthreads();
    Red r;
    red_init<1, 0>(r);
    for (int k = threadIdx.x; k < g; k += kThreads) r.v[0] = r.v[0] + s_slot[k];
    block_reduce<1, 0>(r, s_red);
    if (threadIdx.x == 0) s_f = a * x + b / x + x * x * r.v[0];
    __syncthreads();
    return s_f;
  };
  const double phi = (sqrt(5.0) - 1.0) / 2.0;
  double x1 = hi - phi * (hi - lo);
  double x2 = lo + phi * (hi - lo);
  double f1 = eval(x1);
  double f2 = eval(x2);
  int it = 0;
  while (true) {
    // every thread holds the same scalars; thread 0 decides for all
    if (threadIdx.x == 0) s_go = (fabs(hi - lo) > tol * fmax(1.0, fabs(lo)) && it < maxiter) ? 1 : 0;
    __syncthreads();
    const int go = s_go;
    __syncthreads();
    if (!go) break;
    if (f1 > f2) {
      lo = x1;
      x1 = x2;
      f1 = f2;
      x2 = lo + phi * (hi - lo);
      f2 = eval(x2);
    } else {
      hi = x2;
      x2 = x1;
      f2 = f1;
      x1 = hi - phi * (hi - lo);
      f1 = eval(x1);
    }
    it++;
  }
  if (threadIdx.x == 0) out[0] = (f1 < f2) ? x1 : x2;
}
}  // namespace

int launch_golden_diag(Ctx* c, double a, double b, double lo, double hi, double tol, double* out) {
  const int maxiter = 200;
  if (c->n > 0 && c->n <= kGoldenDeviceMaxN) {
    golden_diag_kernel<<<1, kThreads, 0, c->stream>>>(c->n, red_grid(c->n), c->diag_Q, c->ATdy, c->QATdy, a, b, lo, hi,
                                                      tol, maxiter, c->d_red_out);
    c->launches++;
    HPR_CUDA(c, cudaGetLastError());
    HPR_TRY(fetch_red(c, 1));
    *out = c->h_red_out[0];
    return HPR_OK;
  }
  double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  auto f = [&](double x, double* fx) -> int {
    HPR_TRY(vec_reduce<1, 0>(c, c->n, GoldenF{c->diag_Q, c->ATdy, c->QATdy, x}, 0));
    HPR_TRY(fetch_red(c, 1));
    *fx = a * x + b / x + x * x * c->h_red_out[0];
    return HPR_OK;
  };
  double x1 = hi - phi * (hi - lo);
  double x2 = lo + phi * (hi - lo);
  double f1, f2;
  HPR_TRY(f(x1, &f1));
  HPR_TRY(f(x2, &f2));
  int it = 0;
  while (std::fabs(hi - lo) > tol * std::max(1.0, std::fabs(lo)) && it < maxiter) {
    if (f1 > f2) {
      lo = x1;
      x1 = x2;
      f1 = f2;
      x2 = lo + phi * (hi - lo);
      HPR_TRY(f(x2, &f2));
    } else {
      hi = x2;
      x2 = x1;
      f2 = f1;
      x1 = hi - phi * (hi - lo);
      HPR_TRY(f(x1, &f1));
    }
    it++;
  }
  *out = (f1 < f2) ? x1 : x2;
  return HPR_OK;
}

// do_restart! (algorithm.jl:1130-1166)
int launch_restart(Ctx* c) {
  size_t nb = (size_t)c->n * sizeof(double), mb = (size_t)c->m * sizeof(double);
  HPR_CUDA(c, cudaMemcpyAsync(c->x, c->x_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
  HPR_CUDA(c, cudaMemcpyAsync(c->last_x, c->x_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
  if (c->has_q) {
    HPR_CUDA(c, cudaMemcpyAsync(c->w, c->w_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
    HPR_CUDA(c, cudaMemcpyAsync(c->last_w, c->w_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
  }
  if (c->m > 0) {
    HPR_CUDA(c, cudaMemcpyAsync(c->y, c->y_bar, mb, cudaMemcpyDeviceToDevice, c->stream));
    HPR_CUDA(c, cudaMemcpyAsync(c->last_y, c->y_bar, mb, cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_q) {
      HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, plain(c->ATy_bar), false, false,
                            0));
      HPR_CUDA(c, cudaMemcpyAsync(c->last_ATy, c->ATy_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
      HPR_CUDA(c, cudaMemcpyAsync(c->ATy, c->ATy_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
    }
  }
  if (c->precision != HPR_PREC_FP64 && c->m > 0) {
    const double* y = c->y;
    float* y32 = c->g32_m;
    HPR_TRY(vec_map(c, c->m, [=] __device__(int64_t i) { y32[i] = (float)y[i]; }));
  }
  c->inner = 0;
  return push_state(c);
}

// ---------------------------------------------------------------------------
// Power iteration (power_iteration_A / _Q, eigenvalues.jl:68-196)
// ---------------------------------------------------------------------------
void power_start_vector(std::vector<double>& z, uint64_t seed) {
  uint64_t s = seed;
  for (size_t i = 0; i < z.size(); ++i) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t t = s;
    t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
    t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
    t ^= (t >> 31);
    double u = (double)(t >> 11) * (1.0 / 9007199254740992.0);
    z[i] = (2.0 * u - 1.0) + 1e-8;
  }
}

namespace {

// The power iteration on lambda_max(AA') for small problems, entirely inside
// one CTA: the same steps as power_generic (q = z/|z|, z = A (A' q),
// lambda = <q, z>, err = |z - lambda q| / (|z| + lambda)) with the
// convergence test on the device, so no host round trip per iteration.
// out[0] = lambda, out[1] = iterations run.
__global__ void __launch_bounds__(kEngineThreads, 1)
    fused_power_kernel(FStage<EpiPlain> s_at, FStage<EpiPlain> s_a, double* z, double* q, int64_t m, int maxit,
                       double tol, double* out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(smem_raw)[threadIdx.x >> 5];
  __shared__ double s_red[kMaxRed][kThreads / 32];
  __shared__ double s_b[4];
  double lambda = 1.0;
  int it = 0;
  for (; it < maxit; ++it) {
    Red r;
    red_init<1, 0>(r);
    for (int64_t i = threadIdx.x; i < m; i += blockDim.x) r.v[0] = r.v[0] + z[i] * z[i];
    block_reduce<1, 0>(r, s_red);
    if (threadIdx.x == 0) s_b[0] = sqrt(r.v[0]);
    __syncthreads();
    const double nz = s_b[0];
    for (int64_t i = threadIdx.x; i < m; i += blockDim.x) q[i] = z[i] / nz;
    __syncthreads();
    fused_stage<EpiPlain, HPR_PREC_FP64>(s_at, false, ws);  // ptq = A' q
    fused_stage<EpiPlain, HPR_PREC_FP64>(s_a, false, ws);   // z = A ptq
    red_init<1, 0>(r);
    for (int64_t i = threadIdx.x; i < m; i += blockDim.x) r.v[0] = r.v[0] + q[i] * z[i];
    block_reduce<1, 0>(r, s_red);
    if (threadIdx.x == 0) s_b[1] = r.v[0];
    __syncthreads();
    lambda = s_b[1];
    Red r2;
    red_init<2, 0>(r2);
    for (int64_t i = threadIdx.x; i < m; i += blockDim.x) {
      const double qi = z[i] - lambda * q[i];
      q[i] = qi;
      r2.v[0] = r2.v[0] + qi * qi;
      r2.v[1] = r2.v[1] + z[i] * z[i];
    }
    block_reduce<2, 0>(r2, s_red);
    if (threadIdx.x == 0) s_b[2] = sqrt(r2.v[0]) / (sqrt(r2.v[1]) + lambda);
    __syncthreads();
    if (s_b[2] < tol) break;
  }
  if (threadIdx.x == 0) {
    out[0] = lambda;
    out[1] = (double)it;
  }
}

int power_fused_A(Ctx* c, int maxit, double tol, double* lam) {
  HPR_TRY(prepare_engine(c));
  std::vector<double> hz(c->m);
  power_start_vector(hz, 1);
  HPR_CUDA(c, cudaMemcpyAsync(c->pz, hz.data(), c->m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  auto sat = fstage(c, c->AT, c->planX, c->d_var_start, c->pq, nullptr, plain(c->ptq), plain(c->ptq), true);
  auto sa = fstage(c, c->A, c->planY, c->d_con_start, c->ptq, nullptr, plain(c->pz), plain(c->pz), true);
  HPR_TRY(allow_engine_smem(c, fused_power_kernel));
  fused_power_kernel<<<1, kEngineThreads, kEngineSmem, c->stream>>>(sat, sa, c->pz, c->pq, c->m, maxit, tol,
                                                                     c->d_red_out + 40);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  HPR_CUDA(c, cudaMemcpyAsync(c->h_red_out + 40, c->d_red_out + 40, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  *lam = c->h_red_out[40];
  return HPR_OK;
}

int power_generic(Ctx* c, int64_t len, bool isA, int maxit, double tol, double* lam) {
  std::vector<double> hz(len);
  power_start_vector(hz, 1);
  double *z = c->pz, *q = c->pq, *tq = c->ptq;
  HPR_CUDA(c, cudaMemcpyAsync(z, hz.data(), len * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  double lambda = 1.0;
  int rc = HPR_OK;
  double* out = c->d_red_out;
  for (int it = 0; it < maxit; ++it) {
    // q = z / ||z||
    if ((rc = vec_reduce<1, 0>(c, len, DotF{z, z}, 20)) != HPR_OK) break;
    const double* nzp = out + 20;
    if ((rc = vec_map(c, len, [=] __device__(int64_t i) { q[i] = z[i] / sqrt(*nzp); })) != HPR_OK) break;
    if (isA) {
      if ((rc = engine_launch(c, c->AT, c->planX, c->d_var_start, q, nullptr, plain(tq), false, false, 0)) != HPR_OK)
        break;
      if ((rc = engine_launch(c, c->A, c->planY, c->d_con_start, tq, nullptr, plain(z), false, false, 0)) != HPR_OK)
        break;
    } else {
      if ((rc = qmap(c, q, z, c->ftmp)) != HPR_OK) break;
    }
    if ((rc = vec_reduce<1, 0>(c, len, DotF{q, z}, 21)) != HPR_OK) break;
    const double* lp = out + 21;
    if ((rc = vec_map(c, len, [=] __device__(int64_t i) { q[i] = z[i] - (*lp) * q[i]; })) != HPR_OK) break;
    if ((rc = vec_reduce<2, 0>(c, len, Dot2F{q, q, z, z}, 22)) != HPR_OK) break;
    if ((rc = fetch_red(c, 24)) != HPR_OK) break;
    lambda = c->h_red_out[21];
    double err = std::sqrt(c->h_red_out[22]) / (std::sqrt(c->h_red_out[23]) + lambda);
    if (err < tol) break;
  }
  cudaStreamSynchronize(c->stream);
  *lam = lambda;
  return rc;
}
}  // namespace

// The power iteration on lambda_max(AA') for large problems.  Per iteration
// q = z/|z| is folded into the first product (tq = A'z / |z|), and
// lambda = <q, znew> = <z, znew>/|z| and |znew - lambda q|^2 =
// |znew|^2 - lambda^2 come from reductions in the second product's
// epilogue, so an iteration is two engine launches and one reduction
// finish; the host reads the results once per batch of iterations.  Same
// steps and stopping rule as power_generic.
int power_two_pass_A(Ctx* c, int maxit, double tol, double* lam) {
  const int64_t m = c->m;
  std::vector<double> hz(m);
  power_start_vector(hz, 1);
  double* zb[2] = {c->pz, c->pq};
  HPR_CUDA(c, cudaMemcpyAsync(zb[0], hz.data(), m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  // Result lanes: kBase holds |z|^2 entering a batch; iteration j of the
  // batch leaves |z_new|^2 in kBase+1+2j and <z_old, z_new> in kBase+2+2j.
  // The host reads a whole batch at once and takes the first iteration that
  // meets the tolerance; the iterations queued after it change nothing it
  // reads, so lambda is the one a check after every iteration would give.
  constexpr int kBatch = 8;
  constexpr int kBase = 30;
  static_assert(kBase + 1 + 2 * kBatch <= 64, "result lanes");
  double* out = c->d_red_out;
  const double* zz = zb[0];
  HPR_TRY(vec_reduce<1, 0>(c, m, DotF{zz, zz}, kBase));  // |z0|^2
  double lambda = 1.0;
  int cur = 0, it = 0;
  bool done = false;
  while (!done && it < maxit) {
    const int nb = std::min(kBatch, maxit - it);
    for (int j = 0; j < nb; ++j) {
      EpiScale es{};
      es.out = c->ptq;
      es.nz2 = out + (j == 0 ? kBase : kBase + 1 + 2 * (j - 1));
      HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, zb[(cur + j) & 1], nullptr, es, false, false, 0));
      EpiPow ep{};
      ep.lin_src[0] = ep.cone_src[0] = zb[(cur + j) & 1];
      ep.out = zb[(cur + j + 1) & 1];
      HPR_TRY(engine_launch(c, c->A, c->planY, c->d_con_start, c->ptq, nullptr, ep, false, true, kBase + 1 + 2 * j,
                            true));
    }
    HPR_TRY(fetch_red(c, kBase + 1 + 2 * nb));
    double nz2 = c->h_red_out[kBase];
    for (int j = 0; j < nb && !done; ++j) {
      const double nn2 = c->h_red_out[kBase + 1 + 2 * j], dot = c->h_red_out[kBase + 2 + 2 * j];
      lambda = dot / std::sqrt(nz2);
      const double r2 = std::max(nn2 - lambda * lambda, 0.0);
      const double err = std::sqrt(r2) / (std::sqrt(nn2) + lambda);
      nz2 = nn2;
      ++it;
      if (err < tol) done = true;
    }
    cur = (cur + nb) & 1;
    // the next batch starts from the last |z|^2
    if (!done)
      HPR_CUDA(c, cudaMemcpyAsync(out + kBase, out + kBase + 1 + 2 * (nb - 1), sizeof(double),
                                  cudaMemcpyDeviceToDevice, c->stream));
  }
  *lam = lambda;
  return HPR_OK;
}

int launch_power_A(Ctx* c, int maxit, double tol, double* lam) {
  if (c->m == 0) {
    *lam = 0.0;
    return HPR_OK;
  }
  auto small = [](const Plan& p) { return (int64_t)p.tasks.size() <= kFusedMaxTiles; };
  if (small(c->planX) && small(c->planY) && kEngineSmem <= kSmemOptinMax) return power_fused_A(c, maxit, tol, lam);
  return power_two_pass_A(c, maxit, tol, lam);
}

int launch_power_Q(Ctx* c, int maxit, double tol, double* lam) {
  if (!c->has_q || c->n == 0) {
    *lam = 0.0;
    return HPR_OK;
  }
  return power_generic(c, c->n, false, maxit, tol, lam);
}

// collect_results! unscaling (algorithm.jl:95-102, 1222-1256)
int launch_unscale(Ctx* c, double* hx, double* hy, double* hz, double* hw) {
  const double bs = c->b_scale, cs = c->c_scale;
  const double *xb = c->x_bar, *col = c->col_norm, *zb = c->z_bar, *wb = c->w_bar, *yb = c->y_bar,
               *row = c->row_norm;
  double* t = c->vtmp_n;
  size_t nb = (size_t)c->n * sizeof(double);
  if (hx || (hw && !c->has_q)) {
    HPR_TRY(vec_map(c, c->n, [=] __device__(int64_t i) { t[i] = bs * (xb[i] / col[i]); }));
    if (hx) HPR_TRY(d2h_copy(c, hx, t, nb));
    if (hw && !c->has_q) HPR_TRY(d2h_copy(c, hw, t, nb));
  }
  if (hw && c->has_q) {
    HPR_TRY(vec_map(c, c->n, [=] __device__(int64_t i) { t[i] = bs * (wb[i] / col[i]); }));
    HPR_TRY(d2h_copy(c, hw, t, nb));
  }
  if (hz) {
    HPR_TRY(vec_map(c, c->n, [=] __device__(int64_t i) { t[i] = cs * (zb[i] * col[i]); }));
    HPR_TRY(d2h_copy(c, hz, t, nb));
  }
  if (hy && c->m > 0) {
    double* tm = c->vtmp_m;
    HPR_TRY(vec_map(c, c->m, [=] __device__(int64_t i) { tm[i] = cs * (yb[i] / row[i]); }));
    HPR_TRY(d2h_copy(c, hy, tm, (size_t)c->m * sizeof(double)));
  }
  return HPR_OK;
}

// process_initial_points! (algorithm.jl:2612-2677)
int launch_initial_points(Ctx* c, const double* hx0, const double* hy0) {
  const double bs = c->b_scale, cs = c->c_scale;
  const int64_t n = c->n, m = c->m;
  const bool hq = c->has_q;
  if (hx0) {
    HPR_CUDA(c, cudaMemcpyAsync(c->vtmp_n, hx0, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double *t = c->vtmp_n, *col = c->col_norm;
    double *x = c->x, *xb = c->x_bar, *lx = c->last_x, *w = c->w, *wb = c->w_bar, *lw = c->last_w;
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) {
      double v = t[i] * col[i] / bs;
      x[i] = v;
      xb[i] = v;
      lx[i] = v;
      if (hq) {
        w[i] = v;
        wb[i] = v;
        lw[i] = v;
      }
    }));
  }
  if (hy0) {
    HPR_CUDA(c, cudaMemcpyAsync(c->vtmp_m, hy0, m * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    const double *t = c->vtmp_m, *row = c->row_norm;
    double *y = c->y, *yb = c->y_bar, *ly = c->last_y;
    HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) {
      double v = t[i];
      v = v * row[i] / cs;
      y[i] = v;
      yb[i] = v;
      ly[i] = v;
    }));
    if (m > 0) {
      if (hq) {
        HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, plain(c->ATy_bar), false, false,
                              0));
        HPR_CUDA(c, cudaMemcpyAsync(c->ATy, c->ATy_bar, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        HPR_CUDA(c, cudaMemcpyAsync(c->last_ATy, c->ATy_bar, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream));
      } else {
        HPR_TRY(engine_launch(c, c->AT, c->planX, c->d_var_start, c->y_bar, nullptr, plain(c->ATy), false, false, 0));
      }
    }
    if (hq) HPR_TRY(qmap(c, c->x_bar, c->Qx, c->ftmp));
    const double *xb = c->x_bar, *aty = hq ? c->ATy_bar : c->ATy, *qx = c->Qx, *cc = c->c;
    double* zb = c->z_bar;
    const double sg = c->sigma;
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) {
      double tmp = hq ? (-qx[i] + aty[i] - cc[i]) : (aty[i] - cc[i]);
      double zr = xb[i] + sg * tmp;
      zb[i] = (xb[i] - zr) / sg;
    }));
    if (m > 0) {
      HPR_TRY(engine_launch(c, c->A, c->planY, c->d_con_start, c->x_bar, nullptr, plain(c->Ax), false, false, 0));
      const double *ax = c->Ax, *yy = c->y, *al = c->AL, *au = c->AU;
      double* s = c->s;
      const double f1 = c->lamA * c->sigma;
      HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { s[i] = cmin(cmax(ax[i] - f1 * yy[i], al[i]), au[i]); }));
    }
  }
  if (c->precision != HPR_PREC_FP64 && m > 0) {
    const double* y = c->y;
    float* y32 = c->g32_m;
    HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { y32[i] = (float)y[i]; }));
  }
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

// FP32 / BF16 copies of the scaled A and A' values (hpr_set_precision).
int repack_values(Ctx* c) {
  for (DevCSR* M : {&c->A, &c->AT}) {
    if (M->nnz == 0) continue;
    if (!M->val32) HPR_TRY(dev_alloc_n(c, &M->val32, M->nnz));
    if (!M->val16) HPR_TRY(dev_alloc_n(c, &M->val16, M->nnz));
    const double* v = M->val;
    float* v32 = M->val32;
    __nv_bfloat16* v16 = M->val16;
    HPR_TRY(vec_map(c, M->nnz, [=] __device__(int64_t i) {
      v32[i] = (float)v[i];
      v16[i] = __double2bfloat16(v[i]);
    }));
    ++M->version32;
  }
  HPR_TRY(prepare_engine(c));
  // FP32 gather copies of y (vtmp_m) and x_hat (vtmp_n) are kept by the
  // epilogues; seed them from the current iterates.
  if (c->m > 0) {
    const double* y = c->y;
    float* y32 = c->g32_m;
    HPR_TRY(vec_map(c, c->m, [=] __device__(int64_t i) { y32[i] = (float)y[i]; }));
  }
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

// Algorithmic bytes of one partial iteration (roofline numerator):
//   sum over A, A' of nnz*(value + 4) + 4*(rows+1) + gathered vector once,
//   plus the epilogue streams (x r/w, last_x, c, x_hat w; l, u on boxed
//   variables; y r/w, last_y; AL, AU on linear rows; soc_rhs on cone rows);
//   on the Q path the two Q products and the wider epilogues as listed.
double iteration_bytes(const Ctx* c) {
  double sv = c->precision == HPR_PREC_FP64 ? 8.0 : (c->precision == HPR_PREC_FP32 ? 4.0 : 2.0);
  double sg = c->precision == HPR_PREC_FP64 ? 8.0 : 4.0;
  double nnz = (double)c->A.nnz;
  double m = (double)c->m, n = (double)c->n;
  double nb = (double)(((int64_t)c->h_var_idx.size() > 1) ? c->n_box : c->n);
  double b = 2.0 * nnz * (sv + 4.0) + 4.0 * (m + 1) + 4.0 * (n + 1) + sg * (m + n);
  if (!c->has_q) {
    b += n * 40.0 + nb * 16.0;       // x r/w, last_x, c, x_hat w; l, u
    b += m * 24.0 + (double)c->m_lin * 16.0 + (m - (double)c->m_lin) * 8.0;  // y r/w, last_y; AL, AU; rhs
    if (c->precision != HPR_PREC_FP64) b += (n + m) * 4.0;  // FP32 copies written
    return b;
  }
  // Q path (zxw1, tempv, y, w2 passes): two products with Q per iteration,
  // Q w and Q w_bar.  Low rank: F v (k rows, gathers v, writes k values)
  // then F'(.) (n rows, gathers the k values); a CSR Q (a caller's operator
  // counts as its identity plan) streams Q and gathers v.
  if (c->q_kind == HPR_Q_DIAG_LOWRANK) {
    double nf = (double)c->F.nnz, k = (double)c->F.nrows;
    b += 2.0 * (nf * 12.0 + 4.0 * (k + 1) + 8.0 * n + 8.0 * k);
    b += 2.0 * (nf * 12.0 + 4.0 * (n + 1) + 8.0 * k);
    b += 2.0 * 8.0 * n;  // qdiag read by the zxw1 and tempv passes
  } else {
    b += 2.0 * ((double)c->Q.nnz * 12.0 + 4.0 * (n + 1) + 8.0 * n);
  }
  b += n * 72.0 + nb * 16.0;  // zxw1: x, last_x, c, ATy, w r; l, u; w_bar, Qw, x, x_hat w
  b += n * 32.0;              // tempv: x_hat, Qw, w_bar r; tempv w
  b += n * 56.0;              // w2: w, w_bar, ATy, last_w, last_ATy r; w, ATy w
  if (c->Q_is_diag) b += n * 24.0;  // fact1, fact2, fact
  b += m * 32.0 + (double)c->m_lin * 16.0 + (m - (double)c->m_lin) * 8.0;  // y r/w, last_y, y_bar w; AL, AU; rhs
  if (c->precision != HPR_PREC_FP64) b += (n + m) * 4.0;
  return b;
}


// ---------------------------------------------------------------------------
// Allocation-free residual evaluation (hpr_compute_residuals_noalloc).
//
// Same kernels and reduction order as launch_residuals, but the per-tile
// reduction slots, the per-block partials of the bound check and the result
// lanes live in a file-scope device array instead of the context's
// reduction buffers, and the read-back goes to the caller's stack instead of
// the context's pinned buffer.  Nothing here starts at zero: every slot is
// written by the tile (or finishing warp) that owns it before
// final_reduce_kernel reads it, so the array needs no initialisation and
// carries nothing from one call to the next.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocScratchBytes = (int64_t)2 << 20;  // 2 MiB
constexpr int64_t kNoAllocDoubles = kNoAllocScratchBytes / (int64_t)sizeof(double);
constexpr int64_t kNoAllocOut = 24;  // result lanes at the end of the array
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

std::mutex g_noalloc_mu[kNoAllocMaxDevices];  // one call at a time per device
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch on the current device, looked up once.
int noalloc_scratch(Ctx* c, double** out) {
  double*& p = g_noalloc_ptr[c->device];
  if (!p) {
    void* a = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    if (e != cudaSuccess)
      return set_err(c, HPR_E_CUDA, std::string("cudaGetSymbolAddress(residual scratch): ") + cudaGetErrorString(e));
    p = static_cast<double*>(a);
  }
  *out = p;
  return HPR_OK;
}

// engine_launch with caller-given reduction slots and result lanes.
template <class Epi>
int engine_launch_into(Ctx* c, const DevCSR& M, const Plan& p, const int32_t* cone_start, const double* xin,
                       const Epi& epi, double* slots, double* out) {
  const int nt = (int)p.tasks.size();
  if (nt == 0) {
    HPR_CUDA(c, cudaMemsetAsync(out, 0, Epi::kNRed * sizeof(double), c->stream));
    return HPR_OK;
  }
  // the tiled copy was allocated by hpr_upload; refreshing it allocates nothing
  if (!p.d_tcol || !p.d_tval) return set_err(c, HPR_E_STATE, "engine layout missing (upload incomplete)");
  HPR_TRY(ensure_tiled(c, M, p));
  EngineArgs a;
  a.M = M;
  a.xin = xin;
  a.xin32 = nullptr;
  a.pv = view_of(p, cone_start);
  a.st = c->d_state;
  a.red_slots = slots;
  a.bump_inner = 0;
  launch_engine_prec<Epi, HPR_PREC_FP64>(c, nt, a, epi);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  final_reduce_kernel<Epi::kNRed, Epi::kMaxMask><<<1, kThreads, 0, c->stream>>>(slots, p.nslots(), out);
  c->launches++;
  HPR_CUDA(c, cudaGetLastError());
  return HPR_OK;
}

}  // namespace

int launch_residuals_noalloc(Ctx* c, bool include_bounds, hpr_residuals* r) {
  if (c->device < 0 || c->device >= kNoAllocMaxDevices)
    return set_err(c, HPR_E_UNSUPPORTED, "hpr_compute_residuals_noalloc: device ordinal above 63");
  if (c->precision != HPR_PREC_FP64)
    return set_err(c, HPR_E_UNSUPPORTED, "hpr_compute_residuals_noalloc: needs the FP64 stream (hpr_set_precision 0)");
  const int64_t slots = std::max<int64_t>(std::max<int64_t>(c->planX.nslots(), c->planY.nslots()), kRedGrid);
  const int64_t need = slots * kMaxRed + kNoAllocOut;
  if (need > kNoAllocDoubles)
    return set_err(c, HPR_E_UNSUPPORTED,
                   "hpr_compute_residuals_noalloc: the tile plan needs " + std::to_string(need * 8) +
                       " bytes of reduction scratch; the static scratch holds " +
                       std::to_string(kNoAllocScratchBytes) + " (use hpr_compute_residuals)");
  std::lock_guard<std::mutex> lock(g_noalloc_mu[c->device]);
  double* scratch = nullptr;
  HPR_TRY(noalloc_scratch(c, &scratch));
  double* out = scratch + (kNoAllocDoubles - kNoAllocOut);
  const double bs = c->b_scale, cs = c->c_scale;
  const bool skipq = !c->has_q;
  // lanes of `out`: [0..5] Rd, [8..12] Rp, [16] bounds (as launch_residuals)
  if (!skipq) HPR_TRY(qmap(c, c->x_bar, c->Qx, c->ftmp));
  EpiRd ed{};
  const double* dsrc[5] = {c->c, c->z_bar, c->x_bar, c->col_norm, skipq ? nullptr : c->Qx};
  for (int k = 0; k < 5; ++k) ed.lin_src[k] = ed.cone_src[k] = dsrc[k];
  ed.hasq = skipq ? 0 : 1;
  ed.cs = cs;
  HPR_TRY(engine_launch_into(c, c->AT, c->planX, c->d_var_start, c->y_bar, ed, scratch, out));
  if (c->m > 0) {
    EpiRp ep{};
    const double* psrc[5] = {c->AL, c->AU, c->row_norm, c->y_bar, c->s};
    const double* pcone[5] = {c->soc_rhs_full, nullptr, c->row_norm, c->y_bar, c->s};
    for (int k = 0; k < 5; ++k) {
      ep.lin_src[k] = psrc[k];
      ep.cone_src[k] = pcone[k];
    }
    ep.bs = bs;
    HPR_TRY(engine_launch_into(c, c->A, c->planY, c->d_con_start, c->x_bar, ep, scratch, out + 8));
  }
  if (include_bounds) {
    bounds_box_kernel<<<592, kThreads, 0, c->stream>>>(c->n, c->l, c->u, c->x_bar, c->col_norm, bs, c->dx);
    int64_t nv = (int64_t)c->h_var_idx.size() - 1;
    if (nv > 0)
      bounds_cone_kernel<<<(int)std::min<int64_t>((nv + 127) / 128, 1184), 128, 0, c->stream>>>(
          nv, c->d_var_start, c->x_bar, c->col_norm, bs, c->dx);
    HPR_CUDA(c, cudaGetLastError());
    const int64_t len = c->n;
    vec_reduce_kernel<1, 1, AbsMaxF><<<kRedGrid, kThreads, 0, c->stream>>>(len, AbsMaxF{c->dx}, scratch);
    final_reduce_kernel<1, 1><<<1, kThreads, 0, c->stream>>>(scratch, kRedGrid, out + 16);
    HPR_CUDA(c, cudaGetLastError());
  }
  double h[17];
  HPR_CUDA(c, cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  auto jmax = [](double a, double b) { return (a != a) ? a : ((b != b) ? b : (a > b ? a : b)); };
  double qx_dot = skipq ? 0.0 : h[5];
  r->primal_obj_bar = bs * cs * (h[3] + 0.5 * qx_dot) + c->obj_constant;
  r->dual_obj_bar = bs * cs * (-0.5 * qx_dot + h[4]) + c->obj_constant;
  if (c->m > 0) r->dual_obj_bar += bs * cs * (h[11] + h[12]);
  r->rel_gap_bar = std::fabs(r->primal_obj_bar - r->dual_obj_bar) /
                   (1.0 + std::max(std::fabs(r->primal_obj_bar), std::fabs(r->dual_obj_bar)));
  double qx_inf = skipq ? 0.0 : h[2];
  r->err_Rd_org_bar = h[0] / (1.0 + jmax(jmax(c->norm_c_org, h[1]), qx_inf));
  if (c->m > 0) {
    double denom = 1.0 + jmax(c->norm_b_org, h[10]);
    r->err_Rp_linear_org_bar = c->m_lin > 0 ? h[8] / denom : 0.0;
    r->err_Rp_soc_org_bar = c->m_lin < c->m ? h[9] / denom : 0.0;
    r->err_Rp_org_bar = jmax(h[8], h[9]) / denom;
  } else {
    r->err_Rp_org_bar = r->err_Rp_linear_org_bar = r->err_Rp_soc_org_bar = 0.0;
  }
  if (include_bounds) r->err_Rp_org_bar = jmax(r->err_Rp_org_bar, h[16]);
  r->KKTx_and_gap_org_bar = jmax(jmax(r->err_Rp_org_bar, r->err_Rd_org_bar), r->rel_gap_bar);
  return HPR_OK;
}

}  // namespace hpr
