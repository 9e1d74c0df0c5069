// hpr_epilogues.cuh — the epilogues of the fused engine (one per HPR
// half-step, residual and reduction pass) and the stage descriptors of the
// single-CTA kernels, shared by the host-driven kernels (hpr_kernels.cu) and
// the device-resident solver (hpr_dsolve.cu).  Arithmetic follows the
// reference's operation order (file:line beside each epilogue); the library
// is compiled with -fmad=false so the only fused multiply-adds are the
// explicit fma() calls standing for the reference's `muladd`.
#pragma once

#include "hpr_engine.cuh"

namespace hpr {

// ---------------------------------------------------------------------------
// Halpern factors from the device-resident counter
// (main_update_gpu!, algorithm.jl:2287-2289).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void halpern(const DevState* st, double& H1, double& H2) {
  long long in = *((volatile const long long*)&st->inner);
  H1 = 1.0 / ((double)in + 2.0);
  H2 = 1.0 - H1;
}

// Every epilogue declares kSlots per-row input streams.  The engine stages
// rows [rb, re) of lin_src[k] (linear tiles) or cone_src[k] (cone tiles)
// into shared memory with the tile, and the epilogue reads them through
// `in(k, i)`; inputs that are rarely needed are read from global memory.

// ---------------------------------------------------------------------------
// x half-step without Q: unified_update_zx_kernel_full!/partial!
// (kernels.jl:5955-6063) and the SOC variable projections (kernels.jl:
// 1652-1706); CPU twin unified_update_zx_cpu! (kernels.jl:7672-7812).
// slots: 0 x, 1 last_x, 2 c, 3 l, 4 u
// ---------------------------------------------------------------------------
struct EpiX {
  static constexpr bool kCones = true;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 5;
  static constexpr int kApplySlots = 2;  // cone_apply reads x, last_x
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  double *x, *x_hat, *x_bar, *z_bar, *dx;
  float* x_hat32;
  int full;
  double sigma, H1, H2;
  __device__ void setup(const DevState* st) {
    sigma = st->sigma;
    halpern(st, H1, H2);
  }
  __device__ __forceinline__ void finish(int64_t i, double xi, double lxi, double xb, double zr) {
    double xh = 2.0 * xb - xi;
    double xn = fma(H2, xh, H1 * lxi);
    if (full) {
      dx[i] = xb - xi;
      x_bar[i] = xb;
      z_bar[i] = (xb - zr) / sigma;
    }
    x[i] = xn;
    x_hat[i] = xh;
    if (x_hat32) x_hat32[i] = (float)xh;
  }
  __device__ void linear(int64_t i, double aty, const In& in, Red&) {
    double xi = in(0, i);
    double tmp = aty - in(2, i);
    double zr = xi + sigma * tmp;
    double xb = cmin(cmax(zr, in(3, i)), in(4, i));
    finish(i, xi, in(1, i), xb, zr);
  }
  __device__ double cone_raw(int64_t i, double aty, const In& in, Red&) { return in(0, i) + sigma * (aty - in(2, i)); }
  __device__ void cone_apply(int64_t i, double zr, double t, double ns, bool head, const In& in, Red&) {
    double xb;
    if (ns <= -t) xb = 0.0;
    else if (ns <= t) xb = zr;
    else {
      double pt = (ns + t) / 2.0;
      xb = head ? pt : (pt / ns) * zr;
    }
    finish(i, in(0, i), in(1, i), xb, zr);
  }
};

// ---------------------------------------------------------------------------
// y half-step: unified_update_y_kernel_full!/partial! (kernels.jl:4354-4456)
// and the SOC constraint projections (kernels.jl:4458-5368); CPU twins
// unified_update_y_noQ_cpu! (7817-7952) and update_y_cpu! (7976-8096).
// slots: linear rows 0 y, 1 last_y, 2 AL, 3 AU; cone rows 0 y, 1 last_y,
// 2 soc_rhs (row-aligned)
// ---------------------------------------------------------------------------
struct EpiY {
  static constexpr bool kCones = true;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 4;
  static constexpr int kApplySlots = 2;  // cone_apply reads y, last_y
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  double *y, *y_bar, *s, *dy;
  float* y32;
  int full, ybar_always;
  double f1, f2, H1, H2;
  __device__ void setup(const DevState* st) {
    f1 = st->lamA * st->sigma;
    f2 = 1.0 / f1;
    halpern(st, H1, H2);
  }
  __device__ __forceinline__ void finish(int64_t i, double yi, double lyi, double yb, double sp) {
    double yh = 2.0 * yb - yi;
    double yn = fma(H2, yh, H1 * lyi);
    if (full) {
      s[i] = sp;
      dy[i] = yb - yi;
      y_bar[i] = yb;
    } else if (ybar_always) {
      y_bar[i] = yb;
    }
    y[i] = yn;
    if (y32) y32[i] = (float)yn;
  }
  __device__ void linear(int64_t i, double ax, const In& in, Red&) {
    double yi = in(0, i);
    double sr = ax - f1 * yi;
    double sp = cmin(cmax(sr, in(2, i)), in(3, i));
    double corr = sp - sr;
    double yb = f2 * corr;
    finish(i, yi, in(1, i), yb, sp);
  }
  __device__ double cone_raw(int64_t i, double ax, const In& in, Red&) { return ax - in(2, i) - f1 * in(0, i); }
  __device__ void cone_apply(int64_t i, double sr, double t, double ns, bool head, const In& in, Red&) {
    double sp;
    if (ns <= -t) sp = 0.0;
    else if (ns <= t) sp = sr;
    else {
      double pt = (ns + t) / 2.0;
      sp = head ? pt : (pt / ns) * sr;
    }
    double yb = f2 * (sp - sr);
    finish(i, in(0, i), in(1, i), yb, sp);
  }
};
#ifndef HPR_ENGINE_MINB_Y
#define HPR_ENGINE_MINB_Y HPR_ENGINE_MINB
#endif
template <>
struct EngineMinBlocks<EpiY> {
  static constexpr int value = HPR_ENGINE_MINB_Y;
};

// ---------------------------------------------------------------------------
// Q path, x/w half-step: unified_update_zxw1_kernel_full!/partial!
// (kernels.jl:379-494) with the SOC-with-Q projections (634-1263); CPU twin
// update_zxw1_cpu! (7487-7664).  qdiag != null means the operator
// diag(qdiag) + F'F and `v` is (F'(F w))_i.
// slots: 0 x, 1 last_x, 2 c, 3 ATy, 4 w, 5 l, 6 u
// ---------------------------------------------------------------------------
struct EpiQX {
  static constexpr bool kCones = true;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 7;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  const double *fact1, *fact2, *qdiag;
  double *x, *x_hat, *x_bar, *z_bar, *dx, *w_bar, *Qw;
  int full, diag;
  double sigma, H1, H2, f1s, f2s;
  __device__ void setup(const DevState* st) {
    sigma = st->sigma;
    halpern(st, H1, H2);
    f2s = 1.0 / (1.0 + st->sigma * st->lamQ);
    f1s = 1.0 - f2s;
  }
  __device__ __forceinline__ double qw(int64_t i, double v, const In& in) {
    return qdiag ? qdiag[i] * in(4, i) + v : v;
  }
  __device__ __forceinline__ void finish(int64_t i, const In& in, double xi, double xb, double zr) {
    double xh = 2.0 * xb - xi;
    double xn = fma(H2, xh, H1 * in(1, i));
    double wi = in(4, i);
    w_bar[i] = diag ? fma(fact1[i], wi, fact2[i] * xh) : fma(f1s, wi, f2s * xh);
    if (full) {
      dx[i] = xb - xi;
      x_bar[i] = xb;
      z_bar[i] = (xb - zr) / sigma;
    }
    x[i] = xn;
    x_hat[i] = xh;
  }
  __device__ void linear(int64_t i, double v, const In& in, Red&) {
    double q = qw(i, v, in);
    Qw[i] = q;
    double xi = in(0, i);
    double tmp = -q + in(3, i) - in(2, i);
    double zr = xi + sigma * tmp;
    double xb = cmin(cmax(zr, in(5, i)), in(6, i));
    finish(i, in, xi, xb, zr);
  }
  __device__ double cone_raw(int64_t i, double v, const In& in, Red&) {
    double q = qw(i, v, in);
    Qw[i] = q;
    return in(0, i) + sigma * (-q + in(3, i) - in(2, i));
  }
  __device__ void cone_apply(int64_t i, double zr, double t, double ns, bool head, const In& in, Red&) {
    double xb;
    if (ns <= -t) xb = 0.0;
    else if (ns <= t) xb = zr;
    else {
      double pt = (ns + t) / 2.0;
      xb = head ? pt : (pt / ns) * zr;
    }
    finish(i, in, in(0, i), xb, zr);
  }
};
// (the Q path's x-step holds more state per row: two nonzeros per lane per
// round keep it from spilling)
template <>
struct EngineChunk<EpiQX> {
  static constexpr int value = kChunk < 2 ? kChunk : 2;
};

// tempv = x_hat + sigma (Qw - Q w_bar): compute_tempv_unified_kernel!
// (kernels.jl:4268-4299); CPU update_y_cpu! (kernels.jl:7988-7989).
// slots: 0 x_hat, 1 Qw, 2 w_bar
struct EpiQT {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 3;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  const double* qdiag;
  double* tempv;
  float* tempv32;
  double sigma;
  __device__ void setup(const DevState* st) { sigma = st->sigma; }
  __device__ void linear(int64_t i, double v, const In& in, Red&) {
    double qwb = qdiag ? qdiag[i] * in(2, i) + v : v;
    double tv = in(0, i) + sigma * (in(1, i) - qwb);
    tempv[i] = tv;
    if (tempv32) tempv32[i] = (float)tv;
  }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// w2 half-step: unified_update_w2_kernel_full!/partial! (kernels.jl:
// 5384-5497); CPU update_w2_cpu! (kernels.jl:8100-8185).
// slots: 0 w, 1 w_bar, 2 ATy, 3 last_w, 4 last_ATy
struct EpiW2 {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 5;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  const double* fact;
  double *w, *w_bar, *aty, *aty_bar, *dw, *atdy;
  int full, diag;
  double H1, H2, fs;
  __device__ void setup(const DevState* st) {
    halpern(st, H1, H2);
    fs = st->sigma / (1.0 + st->sigma * st->lamQ);
  }
  __device__ void linear(int64_t i, double ab, const In& in, Red&) {
    double wi = in(0, i), wbi = in(1, i), ai = in(2, i);
    double f = diag ? fact[i] : fs;
    double wbn = wbi + f * (ab - ai);
    double wn = H1 * in(3, i) + H2 * (2.0 * wbn - wi);
    double an = H1 * in(4, i) + H2 * (2.0 * ab - ai);
    w[i] = wn;
    aty[i] = an;
    if (full) {
      w_bar[i] = wbn;
      dw[i] = wbn - wi;
      atdy[i] = ab - ai;
      aty_bar[i] = ab;
    }
  }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// out = M v (+ diag(qdiag) vin for the diag + F'F operator).
struct EpiPlain {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 0;
  using In = Vals<kSlots>;
  const double* lin_src[1];
  const double* cone_src[1];
  double* out;
  const double *qdiag, *vin;
  __device__ void setup(const DevState*) {}
  __device__ void linear(int64_t i, double v, const In&, Red&) { out[i] = qdiag ? qdiag[i] * vin[i] + v : v; }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// out = M v and <out, other>.   slots: 0 other
struct EpiDot {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 1;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 1;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  double* out;
  __device__ void setup(const DevState*) {}
  __device__ void linear(int64_t i, double v, const In& in, Red& r) {
    out[i] = v;
    r.v[0] = r.v[0] + v * in(0, i);
  }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// Power-iteration half-steps (two SpMVs per iteration instead of two SpMVs
// and seven vector kernels):
// out = (M v) / |z|, with |z|^2 read from the device (the normalisation of
// the iterate folded into the first product)
struct EpiScale {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 0;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 0;
  using In = Vals<kSlots>;
  const double* lin_src[1];
  const double* cone_src[1];
  double* out;
  const double* nz2;  // |z|^2
  double inv;
  __device__ void setup(const DevState*) { inv = 1.0 / sqrt(*nz2); }
  __device__ void linear(int64_t i, double v, const In&, Red&) { out[i] = v * inv; }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// out = M v with lanes 0: |out|^2, 1: <zold, out>.   slots: 0 zold
struct EpiPow {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 2;
  static constexpr unsigned kMaxMask = 0;
  static constexpr int kSlots = 1;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  double* out;
  __device__ void setup(const DevState*) {}
  __device__ void linear(int64_t i, double v, const In& in, Red& r) {
    out[i] = v;
    r.v[0] = r.v[0] + v * v;
    r.v[1] = r.v[1] + in(0, i) * v;
  }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};
#ifndef HPR_ENGINE_MINB_POW
#define HPR_ENGINE_MINB_POW HPR_ENGINE_MINB  // CTAs per SM of the power iteration's products
#endif
template <>
struct EngineMinBlocks<EpiScale> {
  static constexpr int value = HPR_ENGINE_MINB_POW;
};
template <>
struct EngineMinBlocks<EpiPow> {
  static constexpr int value = HPR_ENGINE_MINB_POW;
};

// Dual residual in original coordinates: compute_Rd_kernel! /
// compute_Rd_noQ_kernel! (kernels.jl:6467-6512) with the objective dots of
// compute_residuals! (algorithm.jl:113-160).
// lanes: 0 max|Rd|, 1 max|A'y_org|, 2 max|Qx_org|, 3 c'x, 4 z'x, 5 x'Qx
// slots: 0 c, 1 z_bar, 2 x_bar, 3 col_norm, 4 Qx (with Q)
struct EpiRd {
  static constexpr bool kCones = false;
  static constexpr int kNRed = 6;
  static constexpr unsigned kMaxMask = 0x7;
  static constexpr int kSlots = 5;
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  int hasq;
  double cs;
  __device__ void setup(const DevState*) {}
  __device__ void linear(int64_t i, double v, const In& in, Red& r) {
    double cn = in(3, i);
    double ci = in(0, i), zi = in(1, i), xi = in(2, i);
    double c_org = ci * cn * cs;
    double a_org = v * cn * cs;
    double z_org = zi * cn * cs;
    double rd;
    if (hasq) {
      double qx = in(4, i);
      double q_org = qx * cn * cs;
      rd = q_org + c_org - a_org - z_org;
      r.v[2] = nanmax(r.v[2], fabs(q_org));
      r.v[5] = r.v[5] + xi * qx;
    } else {
      rd = c_org - a_org - z_org;
    }
    r.v[0] = nanmax(r.v[0], fabs(rd));
    r.v[1] = nanmax(r.v[1], fabs(a_org));
    r.v[3] = r.v[3] + ci * xi;
    r.v[4] = r.v[4] + zi * xi;
  }
  __device__ double cone_raw(int64_t, double v, const In&, Red&) { return v; }
  __device__ void cone_apply(int64_t, double, double, double, bool, const In&, Red&) {}
};

// Primal residual in original coordinates: compute_Rp_kernel! and
// compute_Rp_SOC_kernel! (kernels.jl:6523-6585) with the dual-objective dots
// y's and y'soc_rhs (algorithm.jl:150-153).
// lanes: 0 max|Rp_lin|, 1 max|Rp_soc|, 2 max|Ax_org|, 3 y's, 4 y'rhs
// slots: linear rows 0 AL, 1 AU, 2 row_norm, 3 y_bar, 4 s;
//        cone rows 0 soc_rhs (row-aligned), 2 row_norm, 3 y_bar, 4 s
struct EpiRp {
  static constexpr bool kCones = true;
  static constexpr int kNRed = 5;
  static constexpr unsigned kMaxMask = 0x7;
  static constexpr int kSlots = 5;
  static constexpr int kApplySlots = 0;  // cone_apply reads no inputs
  using In = Vals<kSlots>;
  const double* lin_src[kSlots];
  const double* cone_src[kSlots];
  double bs;
  __device__ void setup(const DevState*) {}
  __device__ void linear(int64_t i, double v, const In& in, Red& r) {
    double rn = in(2, i);
    double ax = v * rn * bs;
    double lo = in(0, i) * rn * bs;
    double hi = in(1, i) * rn * bs;
    double pr = cmin(cmax(ax, lo), hi);
    double rp = pr - ax;
    r.v[0] = nanmax(r.v[0], fabs(rp));
    r.v[2] = nanmax(r.v[2], fabs(ax));
    r.v[3] = r.v[3] + in(3, i) * in(4, i);
  }
  __device__ double cone_raw(int64_t i, double v, const In& in, Red& r) {
    double rn = in(2, i);
    double ax = v * rn * bs;
    double rh = in(0, i);
    double rt = rh * rn * bs;
    double yb = in(3, i);
    r.v[2] = nanmax(r.v[2], fabs(ax));
    r.v[3] = r.v[3] + yb * in(4, i);
    r.v[4] = r.v[4] + yb * rh;
    return ax - rt;
  }
  __device__ void cone_apply(int64_t i, double sr, double t, double ns, bool head, const In&, Red& r) {
    double rp;
    if (ns <= -t) rp = sr;
    else if (ns <= t) rp = 0.0;
    else if (head) rp = (ns + t) / 2 - t;
    else {
      double f = (1 + t / ns) / 2;
      rp = f * sr - sr;
    }
    r.v[1] = nanmax(r.v[1], fabs(rp));
  }
};


// out = M v (+ diag(qdiag) vin): the plain product epilogue of a stage.
inline EpiPlain plain(double* out, const double* qdiag = nullptr, const double* vin = nullptr) {
  EpiPlain e{};
  e.out = out;
  e.qdiag = qdiag;
  e.vin = vin;
  return e;
}

// Epilogues of one HPR iteration (no-Q: EpiX, EpiY; Q: EpiQX, EpiQT, EpiY,
// EpiW2), set up from the context's workspace.
struct IterEpis {
  EpiY ey{};
  EpiX ex{};
  EpiQX eq{};
  EpiQT et{};
  EpiW2 e2{};
};

inline void make_iter_epis(Ctx* c, bool full, IterEpis& E) {
  const bool fp32 = c->precision != HPR_PREC_FP64;
  if (c->m > 0) {
    EpiY& ey = E.ey;
    const double* ysrc[4] = {c->y, c->last_y, c->AL, c->AU};
    const double* ycone[4] = {c->y, c->last_y, c->soc_rhs_full, nullptr};
    for (int k = 0; k < 4; ++k) {
      ey.lin_src[k] = ysrc[k];
      ey.cone_src[k] = ycone[k];
    }
    ey.y = c->y;
    ey.y_bar = c->y_bar;
    ey.s = c->s;
    ey.dy = c->dy;
    ey.y32 = fp32 ? c->g32_m : nullptr;
    ey.full = full ? 1 : 0;
    ey.ybar_always = c->has_q ? 1 : 0;
  }
  if (!c->has_q) {
    EpiX& ex = E.ex;
    const double* xsrc[5] = {c->x, c->last_x, c->c, c->l, c->u};
    for (int k = 0; k < 5; ++k) {
      ex.lin_src[k] = xsrc[k];
      ex.cone_src[k] = k < 3 ? xsrc[k] : nullptr;
    }
    ex.x = c->x;
    ex.x_hat = c->x_hat;
    ex.x_bar = c->x_bar;
    ex.z_bar = c->z_bar;
    ex.dx = c->dx;
    ex.x_hat32 = fp32 ? c->g32_n : nullptr;
    ex.full = full ? 1 : 0;
    return;
  }
  const bool lowrank = c->q_kind == HPR_Q_DIAG_LOWRANK;
  EpiQX& eq = E.eq;
  const double* qsrc[7] = {c->x, c->last_x, c->c, c->ATy, c->w, c->l, c->u};
  for (int k = 0; k < 7; ++k) {
    eq.lin_src[k] = qsrc[k];
    eq.cone_src[k] = k < 5 ? qsrc[k] : nullptr;
  }
  eq.fact1 = c->fact1;
  eq.fact2 = c->fact2;
  eq.qdiag = lowrank ? c->qdiag : nullptr;
  eq.x = c->x;
  eq.x_hat = c->x_hat;
  eq.x_bar = c->x_bar;
  eq.z_bar = c->z_bar;
  eq.dx = c->dx;
  eq.w_bar = c->w_bar;
  eq.Qw = c->Qw;
  eq.full = full ? 1 : 0;
  eq.diag = c->Q_is_diag ? 1 : 0;
  EpiQT& et = E.et;
  const double* tsrc[3] = {c->x_hat, c->Qw, c->w_bar};
  for (int k = 0; k < 3; ++k) et.lin_src[k] = et.cone_src[k] = tsrc[k];
  et.qdiag = lowrank ? c->qdiag : nullptr;
  et.tempv = c->tempv;
  et.tempv32 = fp32 ? c->g32_n : nullptr;
  EpiW2& e2 = E.e2;
  const double* wsrc[5] = {c->w, c->w_bar, c->ATy, c->last_w, c->last_ATy};
  for (int k = 0; k < 5; ++k) e2.lin_src[k] = e2.cone_src[k] = wsrc[k];
  e2.fact = c->fact;
  e2.w = c->w;
  e2.w_bar = c->w_bar;
  e2.aty = c->ATy;
  e2.aty_bar = c->ATy_bar;
  e2.dw = c->dw;
  e2.atdy = c->ATdy;
  e2.full = full ? 1 : 0;
  e2.diag = c->Q_is_diag ? 1 : 0;
}


// ---------------------------------------------------------------------------
// Stages of the single-CTA kernels: one matrix side, its plan and the
// partial / full epilogues of one half-step.  A problem whose sides have at
// most kFusedMaxTiles tiles runs in one CTA; its warps take the tiles of a
// stage statically, kFusedChunk nonzeros per lane per step.
// ---------------------------------------------------------------------------
#ifndef HPR_FUSED_MAX_TILES
#define HPR_FUSED_MAX_TILES (4 * kWarpsPerCta)
#endif
constexpr int kFusedMaxTiles = HPR_FUSED_MAX_TILES;
#ifndef HPR_FUSED_CHUNK
#define HPR_FUSED_CHUNK 8
#endif
constexpr int kFusedChunk = HPR_FUSED_CHUNK;
template <class E>
struct FStage {
  EngineArgs a;
  E part, full;
  int on;
};

template <class E, int PREC>
__device__ __forceinline__ void fused_stage(const FStage<E>& s, bool last, WarpSmem& ws) {
  if (!s.on) return;
  E e = last ? s.full : s.part;
  e.setup(s.a.st);
  for (int t = threadIdx.x >> 5; t < s.a.pv.ntasks; t += kWarpsPerCta)
    process_warp_tile<E, PREC, true, kFusedChunk>(s.a, e, t, ws);
  __syncthreads();
}

template <class E>
inline FStage<E> fstage(Ctx* c, const DevCSR& M, const Plan& p, const int32_t* cs, const double* xin, const float* xin32,
                 const E& part, const E& full, bool on) {
  FStage<E> s;
  s.a.M = M;
  s.a.xin = xin;
  s.a.xin32 = xin32;
  s.a.pv = view_of(p, cs);
  s.a.st = c->d_state;
  s.a.red_slots = nullptr;
  s.a.bump_inner = 0;
  s.part = part;
  s.full = full;
  s.on = on ? 1 : 0;
  return s;
}

}  // namespace hpr
