// hpr_dsolve.cu — the device-resident solve loop for small problems and the
// request loop of the serving server.
//
// A problem that fits the single-CTA kernels (every matrix side at most
// kFusedMaxTiles tiles, FP64, no Q or a CSR Q) is solved entirely by one CTA:
// the HPR iterations, the residual checks, the restart test, the sigma
// update (with the golden-section search for a diagonal Q), the restarts and
// the termination test of `solve` (algorithm.jl:2765-2905, with
// check_restart 1016-1099, update_sigma! 729-990, do_restart! 1130-1166 and
// compute_residuals! 113-196), with no host round trip.  The scalar logic is
// the host loop's (hpr_api.cu `solve_loop`), run by thread 0; the vector
// work uses the CTA's eight warps, with every reduction in a fixed order, so
// a problem's result does not depend on what runs beside it.
//
// The serving server prepares each request on its own context (upload,
// scaling, power iteration: solve_setup) and hands it to the request loop: a
// persistent kernel whose CTAs take published requests from a device queue,
// solve each one and signal completion through mapped host memory.  A CTA
// that finds no work for kIdleNs exits; the host relaunches the loop when a
// request is waiting and no CTA runs.  Requests that arrive while others
// are solving are taken as soon as a CTA is free, and their work overlaps on
// the device.
#include <algorithm>
#include <atomic>
#include <memory>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

#include "hpr_epilogues.cuh"

namespace hpr {

namespace {

constexpr int kDThreads = kEngineThreads;  // 8 warps, as the single-CTA kernels
static_assert(kDThreads == kThreads, "block reductions assume kThreads threads");

// One prepared request: the views of its context and the solve parameters.
struct DSolve {
  EngineArgs ax, ay, aq;  // A' (X), A (Y), Q with their plans; xin / slots set per use
  IterEpis part, full;    // iteration epilogues (partial / full steps)
  double *x, *x_hat, *x_bar, *last_x, *z_bar, *dx;
  double *y, *y_bar, *last_y, *s, *dy;
  double *w, *w_bar, *last_w, *dw, *Qw, *dQw, *Qx, *tempv;
  double *ATy, *ATy_bar, *last_ATy, *ATdy, *QATdy;
  const double *c, *l, *u, *AL, *AU, *soc_rhs_full, *row_norm, *col_norm;
  const double *diag_Q;
  double *fact1, *fact2, *fact, *fact_M;
  const int32_t* var_start;
  int64_t nvar_cones;
  double* red;  // reduction slots of the context
  DevState* st;
  int64_t n, m, m_lin;
  int has_q, q_diag;
  double b_scale, c_scale, norm_b_org, norm_c_org, obj_constant, lamA, lamQ, sigma0;
  double stoptol, time_limit;
  int64_t max_iter, check_iter, print_frequency;
};

// What the CTA reports (in mapped host memory).
struct DOut {
  int64_t iter, iter_4, iter_6;
  double time, time_4, time_6, sigma_final;
  int32_t status, restarts;
  int32_t error;  // HPR_OK or HPR_E_NUMERIC
  int32_t done;
  hpr_residuals last;
  // seconds of the CTA in: iterations, residual checks, M-norms, sigma
  // updates, restarts; and the number of residual checks
  double t_iter, t_res, t_mnorm, t_sigma, t_restart;
  int64_t checks;
};

struct DCtl {
  int32_t next;       // requests claimed by CTAs
  int32_t published;  // requests published by the host (only grows)
  int32_t pad[30];
};

// ---- block-level primitives (all kDThreads threads call them) --------------

struct BlkShared {
  double red[kMaxRed][kThreads / 32];
  double v[16];  // broadcast scalars
  int go;
};

__device__ __forceinline__ double now_s() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return (double)t * 1e-9;
}

// Fixed-order reduction of NRED lanes over i < n of f(i, r).
template <int NRED, unsigned MASK, class F>
__device__ void blk_reduce(int64_t n, F f, BlkShared& sh, double* out) {
  Red r;
  red_init<NRED, MASK>(r);
  for (int64_t i = threadIdx.x; i < n; i += kDThreads) f(i, r);
  block_reduce<NRED, MASK>(r, sh.red);
  if (threadIdx.x == 0)
    for (int k = 0; k < NRED; ++k) out[k] = r.v[k];
  __syncthreads();
}

template <class F>
__device__ void blk_map(int64_t n, F f) {
  for (int64_t i = threadIdx.x; i < n; i += kDThreads) f(i);
  __syncthreads();
}

// One engine pass over a matrix side: xin gathered, epilogue `e`, reduction
// slots in d.red; with NRED > 0 the slots are then reduced in slot order.
// The pass's arguments live in shared memory (one copy for the CTA, read
// by every warp).  Each pass is a function of its own, so its tile loop
// gets a register allocation of its own instead of sharing one with the
// whole solve loop.
static_assert(sizeof(EngineArgs) % 8 == 0, "EngineArgs copied in 8-byte words");

// dst (shared) = base with xin and the reduction slots set; all threads call
__device__ void blk_args(EngineArgs& dst, const EngineArgs& base, const double* xin, double* slots) {
  constexpr int kWords = (int)(sizeof(EngineArgs) / 8);
  if (threadIdx.x < kWords)
    reinterpret_cast<uint64_t*>(&dst)[threadIdx.x] = reinterpret_cast<const uint64_t*>(&base)[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    dst.xin = xin;
    dst.xin32 = nullptr;
    dst.red_slots = slots;
  }
  __syncthreads();
}

// One pass over prepared (shared-memory) arguments.
template <class E>
__device__ __noinline__ void blk_pass_args(const EngineArgs& a, E e, WarpSmem& ws, BlkShared& sh, double* out);

template <class E>
__device__ void blk_pass(const EngineArgs& base, const double* xin, E e, double* slots, WarpSmem& ws, BlkShared& sh,
                         double* out) {
  __shared__ __align__(16) unsigned char a_raw[sizeof(EngineArgs)];
  EngineArgs& a = *reinterpret_cast<EngineArgs*>(a_raw);
  blk_args(a, base, xin, slots);
  blk_pass_args(a, e, ws, sh, out);
}

template <class E>
__device__ __noinline__ void blk_pass_args(const EngineArgs& a, E e, WarpSmem& ws, BlkShared& sh, double* out) {
  double* slots = a.red_slots;
  e.setup(a.st);
  for (int t = threadIdx.x >> 5; t < a.pv.ntasks; t += kWarpsPerCta)
    process_warp_tile<E, HPR_PREC_FP64, true, kFusedChunk>(a, e, t, ws);
  __syncthreads();
  if constexpr (E::kNRed > 0) {
    const int ns = a.pv.ntasks + a.pv.nbig + a.pv.nlng;
    Red r;
    red_init<E::kNRed, E::kMaxMask>(r);
    for (int q = threadIdx.x; q < ns; q += kDThreads) {
      Red o;
      for (int k = 0; k < E::kNRed; ++k) o.v[k] = __ldcg(slots + (int64_t)q * kMaxRed + k);
      red_combine<E::kNRed, E::kMaxMask>(r, o);
    }
    block_reduce<E::kNRed, E::kMaxMask>(r, sh.red);
    if (threadIdx.x == 0)
      for (int k = 0; k < E::kNRed; ++k) out[k] = r.v[k];
    __syncthreads();
  }
}

__device__ inline EpiPlain plain_epi(double* out) {
  EpiPlain e{};
  e.out = out;
  return e;
}

// Q v (CSR Q; the serving path has no operator Q)
__device__ void blk_qmap(const DSolve& d, const double* v, double* out, WarpSmem& ws, BlkShared& sh) {
  blk_pass(d.aq, v, plain_epi(out), nullptr, ws, sh, nullptr);
}

// The iteration passes' arguments, prepared once per request.
struct IterArgs {
  EngineArgs x, y, qw, qwb;  // no Q: x (A', y), y (A, x_hat); Q: qw, qwb, y (A, tempv), x (A', y_bar)
};

__device__ void blk_iter_args(const DSolve& d, IterArgs& ia) {
  if (!d.has_q) {
    blk_args(ia.x, d.ax, d.y, nullptr);
    blk_args(ia.y, d.ay, d.x_hat, nullptr);
  } else {
    blk_args(ia.qw, d.aq, d.w, nullptr);
    blk_args(ia.qwb, d.aq, d.w_bar, nullptr);
    blk_args(ia.y, d.ay, d.tempv, nullptr);
    blk_args(ia.x, d.ax, d.y_bar, nullptr);
  }
}

// k HPR iterations, the last one full when full_last (the single-CTA
// kernel's loop; thread 0 advances the Halpern counter).
__device__ void blk_iterate(const DSolve& d, const IterArgs& ia, int64_t k, bool full_last, WarpSmem& ws,
                            BlkShared& sh) {
  for (int64_t it = 0; it < k; ++it) {
    const bool last = full_last && it + 1 == k;
    const IterEpis& E = last ? d.full : d.part;
    if (!d.has_q) {
      blk_pass_args(ia.x, E.ex, ws, sh, nullptr);
      if (d.m > 0) blk_pass_args(ia.y, E.ey, ws, sh, nullptr);
    } else {
      blk_pass_args(ia.qw, E.eq, ws, sh, nullptr);
      if (d.m > 0) {
        blk_pass_args(ia.qwb, E.et, ws, sh, nullptr);
        blk_pass_args(ia.y, E.ey, ws, sh, nullptr);
      }
      blk_pass_args(ia.x, E.e2, ws, sh, nullptr);
    }
    if (threadIdx.x == 0) d.st->inner = d.st->inner + 1;
    __syncthreads();
  }
}

// compute_residuals! (algorithm.jl:113-196), as launch_residuals.
__device__ void blk_residuals(const DSolve& d, bool include_bounds, hpr_residuals* rsp, WarpSmem& ws,
                              BlkShared& sh) {
  const double bs = d.b_scale, cs = d.c_scale;
  const bool skipq = !d.has_q;
  __shared__ double h[17];
  if (!skipq) blk_qmap(d, d.x_bar, d.Qx, ws, sh);
  EpiRd ed{};
  const double* dsrc[5] = {d.c, d.z_bar, d.x_bar, d.col_norm, skipq ? nullptr : d.Qx};
  for (int k = 0; k < 5; ++k) ed.lin_src[k] = ed.cone_src[k] = dsrc[k];
  ed.hasq = skipq ? 0 : 1;
  ed.cs = cs;
  blk_pass(d.ax, d.y_bar, ed, d.red, ws, sh, h);
  if (d.m > 0) {
    EpiRp ep{};
    const double* psrc[5] = {d.AL, d.AU, d.row_norm, d.y_bar, d.s};
    const double* pcone[5] = {d.soc_rhs_full, nullptr, d.row_norm, d.y_bar, d.s};
    for (int k = 0; k < 5; ++k) {
      ep.lin_src[k] = psrc[k];
      ep.cone_src[k] = pcone[k];
    }
    ep.bs = bs;
    blk_pass(d.ay, d.x_bar, ep, d.red, ws, sh, h + 8);
  }
  if (include_bounds) {
    // compute_err_lu / compute_err_soc (kernels.jl:6589-6655) into dx
    const double *l = d.l, *u = d.u, *xb = d.x_bar, *col = d.col_norm;
    double* dx = d.dx;
    blk_map(d.n, [&](int64_t i) {
      double lv = cmax(l[i] - xb[i], 0.0);
      double uv = cmax(xb[i] - u[i], 0.0);
      dx[i] = (lv + uv) * (bs / col[i]);
    });
    const int32_t* vs = d.var_start;
    for (int64_t k = threadIdx.x; k < d.nvar_cones; k += kDThreads) {
      const int64_t st = vs[k], en = vs[k + 1];
      const double t = xb[st];
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
        const double f = (1 + t / ns) / 2;
        dx[st] = (ns + t) / 2 - t;
        for (int64_t j = st + 1; j < en; ++j) dx[j] = f * dx[j] - dx[j];
      }
      for (int64_t j = st; j < en; ++j) dx[j] *= bs / col[j];
    }
    __syncthreads();
    blk_reduce<1, 1>(d.n, [&](int64_t i, Red& r) { r.v[0] = nanmax(r.v[0], fabs(dx[i])); }, sh, h + 16);
  }
  if (threadIdx.x == 0) {
    hpr_residuals& r = *rsp;
    auto jmax = [](double a, double b) { return (a != a) ? a : ((b != b) ? b : (a > b ? a : b)); };
    const double qx_dot = skipq ? 0.0 : h[5];
    r.primal_obj_bar = bs * cs * (h[3] + 0.5 * qx_dot) + d.obj_constant;
    r.dual_obj_bar = bs * cs * (-0.5 * qx_dot + h[4]) + d.obj_constant;
    if (d.m > 0) r.dual_obj_bar += bs * cs * (h[11] + h[12]);
    r.rel_gap_bar = fabs(r.primal_obj_bar - r.dual_obj_bar) /
                    (1.0 + cmax(fabs(r.primal_obj_bar), fabs(r.dual_obj_bar)));
    const double qx_inf = skipq ? 0.0 : h[2];
    r.err_Rd_org_bar = h[0] / (1.0 + jmax(jmax(d.norm_c_org, h[1]), qx_inf));
    if (d.m > 0) {
      const double denom = 1.0 + jmax(d.norm_b_org, h[10]);
      r.err_Rp_linear_org_bar = d.m_lin > 0 ? h[8] / denom : 0.0;
      r.err_Rp_soc_org_bar = d.m_lin < d.m ? h[9] / denom : 0.0;
      r.err_Rp_org_bar = jmax(h[8], h[9]) / denom;
    } else {
      r.err_Rp_org_bar = r.err_Rp_linear_org_bar = r.err_Rp_soc_org_bar = 0.0;
    }
    if (include_bounds) r.err_Rp_org_bar = jmax(r.err_Rp_org_bar, h[16]);
    r.KKTx_and_gap_org_bar = jmax(jmax(r.err_Rp_org_bar, r.err_Rd_org_bar), r.rel_gap_bar);
  }
  __syncthreads();
}

// compute_M_norm! (algorithm.jl:1302-1359), as launch_mnorm.
__device__ double blk_mnorm(const DSolve& d, double sg, WarpSmem& ws, BlkShared& sh) {
  const bool skipq = !d.has_q;
  __shared__ double h[8];
  const double *dx = d.dx, *dy = d.dy;
  blk_reduce<1, 0>(d.n, [&](int64_t i, Red& r) { r.v[0] = r.v[0] + dx[i] * dx[i]; }, sh, h + 0);
  if (d.m > 0) blk_reduce<1, 0>(d.m, [&](int64_t i, Red& r) { r.v[0] = r.v[0] + dy[i] * dy[i]; }, sh, h + 1);
  const double *dQw = d.dQw, *dw = d.dw;
  if (!skipq) {
    blk_qmap(d, d.dw, d.dQw, ws, sh);
    blk_reduce<2, 0>(d.n, [&](int64_t i, Red& r) {
      r.v[0] = r.v[0] + dQw[i] * dx[i];
      r.v[1] = r.v[1] + dQw[i] * dQw[i];
    }, sh, h + 3);
  }
  if (d.m > 0) {
    EpiDot e{};
    e.lin_src[0] = e.cone_src[0] = d.dx;
    e.out = d.ATdy;
    blk_pass(d.ax, d.dy, e, d.red, ws, sh, h + 2);
  }
  double M1 = 0.0, M2 = (1.0 / sg) * h[0], M3 = 0.0;
  const double dqw2 = h[4];
  if (!skipq) M2 -= 2.0 * h[3];
  __shared__ double g[2];
  if (d.m > 0) {
    M1 = sg * d.lamA * h[1];
    if (!skipq) {
      blk_qmap(d, d.ATdy, d.QATdy, ws, sh);
      double* atdy = d.ATdy;
      const double* qatdy = d.QATdy;
      blk_reduce<1, 0>(d.n, [&](int64_t i, Red& r) { r.v[0] = r.v[0] + dQw[i] * atdy[i]; }, sh, g);
      M1 -= 2.0 * sg * g[0];
      M2 += 2.0 * h[2];
      if (d.q_diag) {
        const double* fm = d.fact_M;
        blk_map(d.n, [&](int64_t i) { atdy[i] *= fm[i]; });
      }
      blk_reduce<2, 0>(d.n, [&](int64_t i, Red& r) {
        r.v[0] = r.v[0] + atdy[i] * qatdy[i];
        r.v[1] = r.v[1] + dw[i] * dQw[i];
      }, sh, g);
      if (d.q_diag) {
        M3 = g[0];
        M1 += sg * dqw2;
      } else {
        M3 = (sg * sg) / (1.0 + sg * d.lamQ) * g[0];
        M1 += sg * d.lamQ * g[1];
      }
    } else {
      M2 += 2.0 * h[2];
    }
  } else if (!d.q_diag && !skipq) {
    blk_reduce<1, 0>(d.n, [&](int64_t i, Red& r) { r.v[0] = r.v[0] + dw[i] * dQw[i]; }, sh, g);
    M1 = sg * d.lamQ * g[0];
  }
  M2 += cmax(M1, 0.0);
  const double M = cmax(M2, 0.0) + cmax(M3, 0.0);
  return sqrt(M);
}

// update_sigma! inner products (algorithm.jl:787-833), as launch_sigma_terms.
__device__ void blk_sigma_terms(const DSolve& d, double* A, double* B, double* C, double* D, WarpSmem& ws,
                                BlkShared& sh) {
  const bool skipq = !d.has_q;
  const int64_t n = d.n, m = d.m;
  __shared__ double h[8];
  if (!skipq) {
    const double *wb = d.w_bar, *lw = d.last_w;
    double* dw = d.dw;
    blk_map(n, [&](int64_t i) { dw[i] = wb[i] - lw[i]; });
    blk_qmap(d, d.dw, d.dQw, ws, sh);
  }
  {
    const double *a = d.x_bar, *b = d.last_x;
    double* o = d.dx;
    blk_reduce<1, 0>(n, [&](int64_t i, Red& r) {
      const double v = a[i] - b[i];
      o[i] = v;
      r.v[0] = r.v[0] + v * v;
    }, sh, h + 0);
  }
  if (m > 0) {
    const double *a = d.y_bar, *b = d.last_y;
    double* o = d.dy;
    blk_reduce<1, 0>(m, [&](int64_t i, Red& r) {
      const double v = a[i] - b[i];
      o[i] = v;
      r.v[0] = r.v[0] + v * v;
    }, sh, h + 1);
  }
  const double *dQw = d.dQw, *dw = d.dw, *atdy = d.ATdy, *qatdy = d.QATdy;
  if (!skipq && m > 0) {
    const double *a = d.ATy_bar, *b = d.last_ATy;
    double* o = d.ATdy;
    blk_reduce<1, 0>(n, [&](int64_t i, Red& r) {
      const double v = a[i] - b[i];
      o[i] = v;
      r.v[0] = r.v[0] + v * v;
    }, sh, h + 7);
    blk_qmap(d, d.ATdy, d.QATdy, ws, sh);
    blk_reduce<2, 0>(n, [&](int64_t i, Red& r) {
      r.v[0] = r.v[0] + dQw[i] * atdy[i];
      r.v[1] = r.v[1] + atdy[i] * qatdy[i];
    }, sh, h + 2);
  }
  if (!skipq)
    blk_reduce<2, 0>(n, [&](int64_t i, Red& r) {
      r.v[0] = r.v[0] + dQw[i] * dQw[i];
      r.v[1] = r.v[1] + dw[i] * dQw[i];
    }, sh, h + 4);
  double a = 0.0, b = h[0], cc = 0.0, dd = 0.0;
  if (m > 0) a = skipq ? d.lamA * h[1] : d.lamA * h[1] - 2.0 * h[2];
  if (!skipq) {
    if (d.q_diag) {
      const double nq = sqrt(h[4]);
      a += nq * nq;
    } else {
      a += d.lamQ * h[5];
      if (m > 0) {
        cc = h[3];
        dd = d.lamQ;
      }
    }
  }
  *A = a;
  *B = b;
  *C = cc;
  *D = dd;
}

// unified_golden_Q_diag (unified_operations.jl:411-449): the golden-section
// search of a x + b/x + x^2 sum_i ATdy_i QATdy_i / (1 + x q_i) in one CTA.
__device__ double blk_golden_diag(const DSolve& d, double a, double b, double lo, double hi, double tol,
                                  BlkShared& sh) {
  const double *dq = d.diag_Q, *cv = d.ATdy, *dv = d.QATdy;
  __shared__ double f;
  auto eval = [&](double x) {
    blk_reduce<1, 0>(d.n, [&](int64_t i, Red& r) { r.v[0] = r.v[0] + cv[i] * (dv[i] / (1.0 + x * dq[i])); }, sh, &f);
    return a * x + b / x + x * x * f;
  };
  const double phi = (sqrt(5.0) - 1.0) / 2.0;
  double x1 = hi - phi * (hi - lo), x2 = lo + phi * (hi - lo);
  double f1 = eval(x1), f2 = eval(x2);
  for (int it = 0; fabs(hi - lo) > tol * fmax(1.0, fabs(lo)) && it < 200; ++it) {
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
  }
  return (f1 < f2) ? x1 : x2;
}

// golden (kernels.jl:6268-6305) for a general Q: scalar only.
__device__ double golden_scalar(double ap, double bp, double cp, double dp, double lo, double hi, double tol) {
  auto f = [&](double x) { return ap * x + bp / x + cp * (x * x) / (1 + dp * x); };
  const double phi = (sqrt(5.0) - 1.0) / 2.0;
  double a = lo, b = hi, c = b - phi * (b - a), dd = a + phi * (b - a);
  double fc = f(c), fd = f(dd);
  for (int i = 0; i < 200; ++i) {
    if (fd < fc) {
      a = c;
      c = dd;
      fc = fd;
      dd = a + phi * (b - a);
      fd = f(dd);
    } else {
      b = dd;
      dd = c;
      fd = fc;
      c = b - phi * (b - a);
      fc = f(c);
    }
    if ((b - a) < tol) break;
  }
  return 0.5 * (a + b);
}

// do_restart! (algorithm.jl:1130-1166), as launch_restart.
__device__ void blk_restart(const DSolve& d, WarpSmem& ws, BlkShared& sh) {
  {
    const double* xb = d.x_bar;
    double *x = d.x, *lx = d.last_x, *w = d.w, *lw = d.last_w;
    const double* wb = d.w_bar;
    const bool hq = d.has_q;
    blk_map(d.n, [&](int64_t i) {
      x[i] = xb[i];
      lx[i] = xb[i];
      if (hq) {
        w[i] = wb[i];
        lw[i] = wb[i];
      }
    });
  }
  if (d.m > 0) {
    const double* yb = d.y_bar;
    double *y = d.y, *ly = d.last_y;
    blk_map(d.m, [&](int64_t i) {
      y[i] = yb[i];
      ly[i] = yb[i];
    });
    if (d.has_q) {
      blk_pass(d.ax, d.y_bar, plain_epi(d.ATy_bar), nullptr, ws, sh, nullptr);
      const double* ab = d.ATy_bar;
      double *la = d.last_ATy, *a = d.ATy;
      blk_map(d.n, [&](int64_t i) {
        la[i] = ab[i];
        a[i] = ab[i];
      });
    }
  }
}

// unified_update_Q_factors! (unified_operations.jl:484-498), diagonal Q.
__device__ void blk_q_factors(const DSolve& d, double s) {
  if (!d.q_diag || !d.has_q) return;
  const double s2 = s * s;
  const double* dq = d.diag_Q;
  double *f2 = d.fact2, *f = d.fact, *f1 = d.fact1, *fm = d.fact_M;
  blk_map(d.n, [&](int64_t i) {
    const double t2 = 1.0 / (1.0 + s * dq[i]);
    f2[i] = t2;
    f[i] = s * t2;
    f1[i] = s * dq[i] * t2;
    fm[i] = s2 * t2;
  });
}

__device__ double jl_clamp(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

// print schedule of the reference (print_step, algorithm.jl): every
// max(10^(floor(log10 iter) - 1), 10) iterations
__device__ bool is_print_iter(int64_t iter, const DSolve& d) {
  if (d.print_frequency != -1) return iter % d.print_frequency == 0 || iter == d.max_iter;
  int64_t p = 1;
  while (p * 10 <= iter) p *= 10;  // 10^floor(log10 iter) (1 for iter < 10)
  int64_t step = p / 10;
  if (step < 10) step = 10;
  return iter % step == 0 || iter == d.max_iter;
}

// The scalar state of the loop (thread 0 owns it; the others read it from
// shared memory after a barrier).
struct LoopState {
  double sigma;
  int flag;
  bool first;
  double last_gap, current_gap, save_gap;
  int64_t inner;
  int times;
  double best_gap, best_kkt, best_sigma;
  int64_t best_iter;
  bool corr_active;
  int corr_dir;
};

// check_restart (algorithm.jl:1016-1099) with should_refresh_best_sigma
// (690-703); thread 0.
__device__ void check_restart(LoopState& R, int64_t iter, int64_t ci, double sigma, double kkt) {
  R.flag = 0;
  if (R.first) {
    if (iter == ci) {
      R.first = false;
      R.flag = 1;
      R.best_gap = R.current_gap;
      R.best_kkt = kkt;
      R.best_sigma = sigma;
    }
    return;
  }
  if (iter % ci != 0) return;
  if (R.current_gap < 0) R.current_gap = 1e-6;
  if (R.current_gap <= 0.36 * R.last_gap) R.flag = 1;
  if (R.current_gap <= 0.8 * R.last_gap && R.current_gap > R.save_gap) R.flag = 2;
  if ((R.inner >= cmax(500.0, 0.15 * (double)iter) || (R.inner >= 10000 && R.current_gap <= 0.75 * R.last_gap)) &&
      R.current_gap > 0.9 * R.save_gap)
    R.flag = 3;
  const bool improved = kkt < R.best_kkt;
  const bool compat = R.current_gap < R.best_gap && kkt <= 1.01 * R.best_kkt;
  const bool periodic = R.best_iter >= 10 && kkt <= 1.2 * R.best_kkt;
  if (improved || compat || periodic) {
    R.best_gap = R.current_gap;
    R.best_kkt = kkt;
    R.best_sigma = sigma;
    R.best_iter = 0;
  }
  R.save_gap = R.current_gap;
}

// update_sigma! (algorithm.jl:729-990): the new sigma from the terms; thread 0.
__device__ double sigma_rule(LoopState& R, const hpr_residuals& res, double sm, double s_old) {
  const double ck = res.KKTx_and_gap_org_bar, cg = R.current_gap;
  const bool ref_ok = (ck <= 10.0 * R.best_kkt) && (cg <= 10.0 * R.best_gap);
  const double pr = jl_clamp(sqrt((ck / R.best_kkt) * (cg / R.best_gap)), 1.0, 10.0);
  double base = sm;
  if (ref_ok) {
    const double th = jl_clamp(exp(-0.3 * (pr - 1.0)), 0.0, 1.0);
    base = jl_clamp(exp(th * log(sm) + (1.0 - th) * log(R.best_sigma)), 1e-12, 1e12);
  }
  const double THR = 1e-8;
  const double ep = cmax(res.err_Rp_org_bar, 1e-16), ed = cmax(res.err_Rd_org_bar, 1e-16);
  const double es = cmin(ep, ed), el = cmax(ep, ed), ir = el / es;
  const bool both = el <= THR;
  const bool one = es <= 0.5 * THR && el >= 2.0 * THR;
  const bool ext = ir >= 1e6;
  const bool trig = !both && (one || ext);
  const bool keep = !both && (es <= 0.8 * THR || ir >= 1e5);
  if (!both && (trig || (R.corr_active && keep))) {
    R.corr_active = true;
    R.corr_dir = ed >= ep ? 1 : -1;
  } else {
    R.corr_active = false;
    R.corr_dir = 0;
  }
  double beta = 0.0;
  if (!both) {
    if (one) beta = 0.5;
    if (ext) beta = 1.0;
    else if (R.corr_active) beta = 0.5;
  }
  double kappa = 1.0;
  if (beta > 0.0) {
    double rk = ed / ep;
    if (R.corr_active) rk = R.corr_dir > 0 ? cmax(rk, 2.0) : cmin(rk, 0.5);
    kappa = exp(beta * jl_clamp(log(rk), -log(100.0), log(100.0)));
  }
  double sn = base * kappa;
  if (R.corr_active) sn = R.corr_dir > 0 ? cmax(sn, s_old * 1.5) : cmin(sn, s_old / 1.5);
  sn = jl_clamp(sn, 1e-12, 1e12);
  R.best_iter += 1;
  return sn;
}

constexpr double kInfD = (double)INFINITY;

// The whole solve loop of one request (solve_loop in hpr_api.cu, from the
// first residual check to termination), by one CTA.
__device__ void dsolve_run(const DSolve& d, DOut* out, double t_start, WarpSmem& ws, BlkShared& sh) {
  __shared__ LoopState R;
  __shared__ hpr_residuals rs;
  __shared__ int64_t s_iter, s_next, iter_4, iter_6;
  __shared__ double time_4, time_6;
  __shared__ int status, s_check, s_err;
  __shared__ double tp[5];  // phase seconds (see DOut)
  // (raw storage: shared variables are not constructed)
  __shared__ __align__(16) unsigned char ia_raw[sizeof(IterArgs)];
  IterArgs& ia = *reinterpret_cast<IterArgs*>(ia_raw);
  blk_iter_args(d, ia);
  __shared__ int64_t n_checks;
  const int64_t ci = d.check_iter;
  auto mark = [&](int k, double t0) {
    if (threadIdx.x == 0) tp[k] += now_s() - t0;
  };
  if (threadIdx.x == 0) {
    R.sigma = d.sigma0;
    R.flag = 0;
    R.first = true;
    R.last_gap = R.current_gap = R.save_gap = kInfD;
    R.inner = 0;
    R.times = 0;
    R.best_gap = R.best_kkt = kInfD;
    R.best_sigma = d.sigma0;
    R.best_iter = 0;
    R.corr_active = false;
    R.corr_dir = 0;
    memset(&rs, 0, sizeof(rs));
    s_iter = 0;
    iter_4 = iter_6 = 0;
    time_4 = time_6 = 0.0;
    status = -1;
    s_err = 0;
    for (int k = 0; k < 5; ++k) tp[k] = 0.0;
    n_checks = 0;
  }
  __syncthreads();
  while (true) {
    // ---- the event iteration (residual check or print)
    if (threadIdx.x == 0) {
      const double el = now_s() - t_start;
      const bool print_yes = is_print_iter(s_iter, d) || el > d.time_limit;
      s_check = (s_iter % ci == 0 || print_yes) ? 1 : 0;
    }
    __syncthreads();
    if (s_check) {
      const double t0 = now_s();
      blk_residuals(d, s_iter == 0, &rs, ws, sh);
      mark(1, t0);
      if (threadIdx.x == 0) ++n_checks;
    }
    if (threadIdx.x == 0) {
      const double kkt = rs.KKTx_and_gap_org_bar;
      if (kkt != kkt) s_err = HPR_E_NUMERIC;
      else if (kkt < d.stoptol) status = HPR_STATUS_OPTIMAL;
      else if (s_iter == d.max_iter) status = HPR_STATUS_MAX_ITER;
      else if (now_s() - t_start > d.time_limit) status = HPR_STATUS_TIME_LIMIT;
      if (!s_err) check_restart(R, s_iter, ci, R.sigma, kkt);
    }
    __syncthreads();
    if (s_err) break;
    // ---- sigma update (update_sigma!, algorithm.jl:729-990)
    const double t_sig = now_s();
    if (R.flag >= 1) {
      __shared__ double ta, tb, tc, td, s_sm;
      double a, b, cc, dd;
      blk_sigma_terms(d, &a, &b, &cc, &dd, ws, sh);
      if (threadIdx.x == 0) {
        ta = cmax(a, 1e-16);
        tb = cmax(b, 1e-16);
        tc = cc;
        td = dd;
      }
      __syncthreads();
      double sm;
      if (!d.has_q || d.m == 0) sm = sqrt(tb / ta);
      else if (d.q_diag) sm = blk_golden_diag(d, ta, tb, 1e-12, 1e12, 1e-13, sh);
      else sm = golden_scalar(ta, tb, tc, td, 1e-12, 1e12, 1e-13);
      if (threadIdx.x == 0) {
        const double s_old = R.sigma;
        const double sn = sigma_rule(R, rs, sm, s_old);
        s_sm = (d.q_diag && d.has_q && fabs(s_old - sn) > 1e-15) ? 1.0 : 0.0;
        R.sigma = sn;
        d.st->sigma = sn;
      }
      __syncthreads();
      if (s_sm != 0.0) blk_q_factors(d, R.sigma);
    }
    mark(3, t_sig);
    if (R.flag > 0) {
      const double t_rs = now_s();
      blk_restart(d, ws, sh);
      mark(4, t_rs);
      if (threadIdx.x == 0) {
        R.last_gap = R.current_gap;
        R.save_gap = kInfD;
        R.times++;
        R.inner = 0;
        d.st->inner = 0;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      const double kkt = rs.KKTx_and_gap_org_bar;
      const double el = now_s() - t_start;
      if (kkt < 1e-4 && iter_4 == 0 && time_4 == 0) {
        time_4 = el;
        iter_4 = s_iter;
        if (s_iter == 0) time_4 = 1e-300;
      }
      if (kkt < 1e-6 && iter_6 == 0 && time_6 == 0) {
        time_6 = el;
        iter_6 = s_iter;
        if (s_iter == 0) time_6 = 1e-300;
      }
      int64_t next = s_iter + 1;
      while (!(next % ci == 0 || is_print_iter(next, d))) ++next;
      s_next = next;
    }
    __syncthreads();
    if (status >= 0) break;
    // ---- steps up to the next event (perform_iteration_step!)
    const int64_t next = s_next;
    int64_t iter = s_iter;
    if (R.flag > 0) {
      double t0 = now_s();
      blk_iterate(d, ia, 1, true, ws, sh);
      mark(0, t0);
      t0 = now_s();
      const double mn = blk_mnorm(d, R.sigma, ws, sh);
      mark(2, t0);
      if (threadIdx.x == 0) {
        R.last_gap = cmin(mn, R.last_gap);
        if ((iter + 1) % ci == 0) R.current_gap = mn;
        R.inner += 1;
      }
      iter += 1;
      if (iter < next) {
        t0 = now_s();
        blk_iterate(d, ia, next - iter, true, ws, sh);
        mark(0, t0);
        if (threadIdx.x == 0) R.inner += next - iter;
        if (next % ci == 0) {
          t0 = now_s();
          const double m2 = blk_mnorm(d, R.sigma, ws, sh);
          mark(2, t0);
          if (threadIdx.x == 0) R.current_gap = m2;
        }
      }
    } else {
      double t0 = now_s();
      blk_iterate(d, ia, next - iter, true, ws, sh);
      mark(0, t0);
      if (threadIdx.x == 0) R.inner += next - iter;
      if (next % ci == 0) {
        t0 = now_s();
        const double m2 = blk_mnorm(d, R.sigma, ws, sh);
        mark(2, t0);
        if (threadIdx.x == 0) R.current_gap = m2;
      }
    }
    if (threadIdx.x == 0) s_iter = next;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double tt = now_s() - t_start;
    out->iter = s_iter;
    out->time = tt;
    out->status = status;
    out->restarts = R.times;
    out->error = s_err;
    out->time_4 = time_4 == 0.0 ? tt : (time_4 < 1e-200 ? 0.0 : time_4);
    out->iter_4 = (iter_4 == 0 && time_4 == 0.0) ? s_iter : iter_4;
    out->time_6 = time_6 == 0.0 ? tt : (time_6 < 1e-200 ? 0.0 : time_6);
    out->iter_6 = (iter_6 == 0 && time_6 == 0.0) ? s_iter : iter_6;
    out->sigma_final = R.sigma;
    out->last = rs;
    out->t_iter = tp[0];
    out->t_res = tp[1];
    out->t_mnorm = tp[2];
    out->t_sigma = tp[3];
    out->t_restart = tp[4];
    out->checks = n_checks;
  }
}

constexpr uint64_t kIdleNs = 200ull * 1000ull * 1000ull;  // a CTA without work exits after 200 ms

__device__ __forceinline__ int ld_acquire_gpu(const int32_t* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The request loop: each CTA claims published requests one at a time
// (claims only ever cover published entries), solves them and marks them
// done in host memory.  The host copies each descriptor and then the new
// published count into device memory; a CTA polls the count with a growing
// pause (1 to 64 us) and exits after kIdleNs without a request.
__global__ void __launch_bounds__(kDThreads, 1)
    request_loop_kernel(const DSolve* __restrict__ reqs, DOut* outs, DCtl* ctl, int cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem& ws = reinterpret_cast<WarpSmem*>(smem_raw)[threadIdx.x >> 5];
  __shared__ BlkShared sh;
  __shared__ int s_req;
  while (true) {
    if (threadIdx.x == 0) {
      s_req = -1;
      const uint64_t t0 = (uint64_t)(now_s() * 1e9);
      unsigned pause = 1000;
      while (true) {
        const int pub = ld_acquire_gpu(&ctl->published);
        const int nx = *((volatile int32_t*)&ctl->next);
        if (nx < pub) {
          if (atomicCAS(&ctl->next, nx, nx + 1) == nx) {
            s_req = nx;
            break;
          }
          continue;
        }
        if ((uint64_t)(now_s() * 1e9) - t0 > kIdleNs) break;
        __nanosleep(pause);
        pause = pause < 64000 ? 2 * pause : pause;
      }
      __threadfence();
    }
    __syncthreads();
    const int r = s_req;
    if (r < 0) return;
    const int slot = r % cap;
    DOut* o = outs + slot;
    dsolve_run(reqs[slot], o, now_s(), ws, sh);
    if (threadIdx.x == 0) {
      __threadfence_system();
      *((volatile int32_t*)&o->done) = 1;
      __threadfence_system();
    }
    __syncthreads();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
bool dsolve_eligible(const Ctx* c, const hpr_params* P) {
  if (P->precision != HPR_PREC_FP64 || P->auto_save) return false;
  if (c->q_kind == HPR_Q_DIAG_LOWRANK || c->q_kind == HPR_Q_OPERATOR) return false;
  auto fits = [](const Plan& p) { return (int64_t)p.tasks.size() <= kFusedMaxTiles; };
  if (!fits(c->planX) || !fits(c->planY)) return false;
  if (c->has_q && !fits(c->planQ)) return false;
  return kEngineSmem <= 48 * 1024;
}

struct DQueue {
  int device = 0;
  int ctas = 0;
  int cap = 0;
  cudaStream_t stream = nullptr;   // the request loop
  cudaStream_t copies = nullptr;   // descriptor uploads
  DSolve* d_reqs = nullptr;
  DCtl* d_ctl = nullptr;
  DOut* h_outs = nullptr;          // mapped host memory
  DOut* d_outs = nullptr;
  int32_t* h_stage = nullptr;      // pinned staging of the published count
  int64_t published = 0;
  std::mutex mu;
  std::vector<uint8_t> busy;       // slot in use (published, result not yet read)
  bool running = false;
  std::string err;
};

namespace {
int q_err(DQueue* q, const std::string& m) {
  q->err = m;
  return HPR_E_CUDA;
}
#define DQ_CUDA(q, call)                                                        \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      (void)cudaGetLastError();                                                 \
      return q_err((q), std::string(#call) + ": " + cudaGetErrorString(e_));    \
    }                                                                           \
  } while (0)

// (re)launch the request loop when no CTA of it runs; called with q->mu held
int ensure_running(DQueue* q) {
  if (q->running) {
    cudaError_t s = cudaStreamQuery(q->stream);
    if (s == cudaErrorNotReady) return HPR_OK;
    if (s != cudaSuccess) return q_err(q, std::string("request loop: ") + cudaGetErrorString(s));
    q->running = false;
  }
  request_loop_kernel<<<q->ctas, kDThreads, kEngineSmem, q->stream>>>(q->d_reqs, q->d_outs, q->d_ctl, q->cap);
  DQ_CUDA(q, cudaGetLastError());
  q->running = true;
  return HPR_OK;
}
}  // namespace

DQueue* dqueue_create(int device, int ctas, int cap, std::string* err) {
  std::unique_ptr<DQueue> q(new DQueue);
  q->device = device;
  q->cap = cap;
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return nullptr;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice failed");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  q->ctas = ctas > 0 ? ctas : sms;
  if (cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&q->copies, cudaStreamNonBlocking) != cudaSuccess)
    return fail("stream creation failed");
  if (cudaMalloc(&q->d_reqs, sizeof(DSolve) * cap) != cudaSuccess || cudaMalloc(&q->d_ctl, sizeof(DCtl)) != cudaSuccess)
    return fail("device memory for the request queue");
  if (cudaMemset(q->d_ctl, 0, sizeof(DCtl)) != cudaSuccess) return fail("cudaMemset");
  if (cudaHostAlloc(&q->h_outs, sizeof(DOut) * cap, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostAlloc(&q->h_stage, 64, cudaHostAllocDefault) != cudaSuccess)
    return fail("pinned host memory for the request queue");
  std::memset(q->h_outs, 0, sizeof(DOut) * cap);
  if (cudaHostGetDevicePointer(&q->d_outs, q->h_outs, 0) != cudaSuccess) return fail("cudaHostGetDevicePointer");
  if (cudaFuncSetAttribute(request_loop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kEngineSmem) !=
      cudaSuccess)
    return fail("request loop attributes");
  q->busy.assign(cap, 0);
  return q.release();
}

void dqueue_destroy(DQueue* q) {
  if (!q) return;
  cudaSetDevice(q->device);
  // the loop ends by itself once idle
  if (q->stream) cudaStreamSynchronize(q->stream);
  if (q->d_reqs) cudaFree(q->d_reqs);
  if (q->d_ctl) cudaFree(q->d_ctl);
  if (q->h_outs) cudaFreeHost(q->h_outs);
  if (q->h_stage) cudaFreeHost(q->h_stage);
  if (q->stream) cudaStreamDestroy(q->stream);
  if (q->copies) cudaStreamDestroy(q->copies);
  delete q;
}

const char* dqueue_error(DQueue* q) { return q ? q->err.c_str() : ""; }

// Build the request from the context (after solve_setup) and publish it;
// *slot_out identifies it for dqueue_poll.
int dqueue_submit(DQueue* q, Ctx* c, const hpr_params* P, double sigma0, int* slot_out) {
  DSolve d = DSolve();
  auto args = [&](const DevCSR& M, const Plan& p, const int32_t* cs) {
    EngineArgs a = EngineArgs();
    a.M = M;
    a.pv = view_of(p, cs);
    a.st = c->d_state;
    return a;
  };
  d.ax = args(c->AT, c->planX, c->d_var_start);
  d.ay = args(c->A, c->planY, c->d_con_start);
  if (c->has_q) d.aq = args(c->Q, c->planQ, c->d_var_start);
  make_iter_epis(c, false, d.part);
  make_iter_epis(c, true, d.full);
  d.x = c->x;
  d.x_hat = c->x_hat;
  d.x_bar = c->x_bar;
  d.last_x = c->last_x;
  d.z_bar = c->z_bar;
  d.dx = c->dx;
  d.y = c->y;
  d.y_bar = c->y_bar;
  d.last_y = c->last_y;
  d.s = c->s;
  d.dy = c->dy;
  d.w = c->w;
  d.w_bar = c->w_bar;
  d.last_w = c->last_w;
  d.dw = c->dw;
  d.Qw = c->Qw;
  d.dQw = c->dQw;
  d.Qx = c->Qx;
  d.tempv = c->tempv;
  d.ATy = c->ATy;
  d.ATy_bar = c->ATy_bar;
  d.last_ATy = c->last_ATy;
  d.ATdy = c->ATdy;
  d.QATdy = c->QATdy;
  d.c = c->c;
  d.l = c->l;
  d.u = c->u;
  d.AL = c->AL;
  d.AU = c->AU;
  d.soc_rhs_full = c->soc_rhs_full;
  d.row_norm = c->row_norm;
  d.col_norm = c->col_norm;
  d.diag_Q = c->diag_Q;
  d.fact1 = c->fact1;
  d.fact2 = c->fact2;
  d.fact = c->fact;
  d.fact_M = c->fact_M;
  d.var_start = c->d_var_start;
  d.nvar_cones = (int64_t)c->h_var_idx.size() - 1;
  d.red = c->d_red;
  d.st = c->d_state;
  d.n = c->n;
  d.m = c->m;
  d.m_lin = c->m_lin;
  d.has_q = c->has_q ? 1 : 0;
  d.q_diag = c->Q_is_diag ? 1 : 0;
  d.b_scale = c->b_scale;
  d.c_scale = c->c_scale;
  d.norm_b_org = c->norm_b_org;
  d.norm_c_org = c->norm_c_org;
  d.obj_constant = c->obj_constant;
  d.lamA = c->lamA;
  d.lamQ = c->lamQ;
  d.sigma0 = sigma0;
  d.stoptol = P->stoptol;
  d.time_limit = P->time_limit;
  d.max_iter = P->max_iter;
  d.check_iter = P->check_iter;
  d.print_frequency = P->print_frequency;
  // the reduction slots must cover every side's plan
  const int64_t need = (int64_t)std::max({c->planX.nslots(), c->planY.nslots(), c->has_q ? c->planQ.nslots() : 0}) *
                       kMaxRed;
  if (need > c->red_slots) return set_err(c, HPR_E_STATE, "reduction slots too small for the device-resident solve");
  // every kernel of the context's setup has finished before the loop reads
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));

  // publication k goes to slot k % cap (the loop claims in publication
  // order); a slot is reused once its previous request has been read
  int slot = -1;
  {
    std::unique_lock<std::mutex> lk(q->mu);
    while (true) {
      slot = (int)(q->published % q->cap);
      if (!q->busy[slot]) break;
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(50));
      lk.lock();
    }
    q->busy[slot] = 1;
    q->h_outs[slot].done = 0;
    // the descriptor, then the count that publishes it, in stream order
    q->published += 1;
    *q->h_stage = (int32_t)q->published;
    HPR_CUDA(c, cudaMemcpyAsync(q->d_reqs + slot, &d, sizeof(DSolve), cudaMemcpyHostToDevice, q->copies));
    HPR_CUDA(c, cudaMemcpyAsync(&q->d_ctl->published, q->h_stage, sizeof(int32_t), cudaMemcpyHostToDevice,
                                q->copies));
    HPR_CUDA(c, cudaStreamSynchronize(q->copies));
    if (ensure_running(q) != HPR_OK) {
      q->busy[slot] = 0;
      return set_err(c, HPR_E_CUDA, q->err);
    }
  }
  *slot_out = slot;
  return HPR_OK;
}

// Relaunch the request loop if it went idle while requests wait (the loop's
// CTAs exit after kIdleNs without work); call it every few milliseconds
// while requests are in flight.
int dqueue_keepalive(DQueue* q) {
  std::unique_lock<std::mutex> lk(q->mu);
  return ensure_running(q);
}

// Non-blocking: when the request in `slot` is done, fill `out` (scalars; the
// solution stays on the context), free the slot and set *done.
int dqueue_poll(DQueue* q, Ctx* c, int slot, hpr_results* out, bool* done) {
  volatile DOut* o = q->h_outs + slot;
  *done = false;
  if (o->done == 0) return HPR_OK;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  DOut r;
  std::memcpy(&r, (const void*)o, sizeof(DOut));
  {
    std::unique_lock<std::mutex> lk(q->mu);
    q->busy[slot] = 0;
  }
  *done = true;
  if (r.error == HPR_E_NUMERIC)
    return set_err(c, HPR_E_NUMERIC, "NaN in the KKT residuals at iteration " + std::to_string(r.iter));
  out->iter = r.iter;
  out->iter_4 = r.iter_4;
  out->iter_6 = r.iter_6;
  out->time = r.time;
  out->time_4 = r.time_4;
  out->time_6 = r.time_6;
  out->status = r.status;
  out->restarts = r.restarts;
  out->sigma_final = r.sigma_final;
  out->last = r.last;
  out->residuals = r.last.KKTx_and_gap_org_bar;
  out->primal_obj = r.last.primal_obj_bar;
  out->gap = r.last.rel_gap_bar;
  c->sigma = r.sigma_final;
  c->dloop[0] = r.t_iter;
  c->dloop[1] = r.t_res;
  c->dloop[2] = r.t_mnorm;
  c->dloop[3] = r.t_sigma;
  c->dloop[4] = r.t_restart;
  c->dloop[5] = (double)r.checks;
  return HPR_OK;
}

// Publish and wait (polls back off to 0.5 ms, so many waiting threads cost
// little CPU).
int dqueue_solve(DQueue* q, Ctx* c, const hpr_params* P, double sigma0, hpr_results* out) {
  int slot = -1;
  HPR_TRY(dqueue_submit(q, c, P, sigma0, &slot));
  int pause_us = 20;
  auto t_last = std::chrono::steady_clock::now();
  for (;;) {
    bool done = false;
    HPR_TRY(dqueue_poll(q, c, slot, out, &done));
    if (done) return HPR_OK;
    std::this_thread::sleep_for(std::chrono::microseconds(pause_us));
    pause_us = std::min(2 * pause_us, 500);
    const auto now = std::chrono::steady_clock::now();
    if (now - t_last > std::chrono::milliseconds(2)) {
      t_last = now;
      if (dqueue_keepalive(q) != HPR_OK) return set_err(c, HPR_E_CUDA, q->err);
    }
  }
}

}  // namespace hpr
