// hpr_scale.cu — Ruiz / SOC block aggregation / Pock–Chambolle / b-c scaling
// on the device (scaling!, src/utils/scaling.jl:785-1289) and
// check_Q_diagonal (scaling.jl:1327-1353).
//
// Every per-element operation follows the reference's GPU kernels
// (kernels.jl:6699-7239): norms are clamped to [1e-4, 1e4] after the sqrt and
// again after SOC block aggregation; A and A' are scaled separately as
// v * (1/r_i) / c_j; Q is scaled as DC^-1 Q DC^-1 and by b_scale/c_scale.
#include <algorithm>
#include <cmath>

#include "hpr_engine.cuh"

namespace hpr {

namespace {

constexpr int PH_RUIZ = 1, PH_PRE_POCK = 2, PH_POCK = 3;
constexpr int LOC_CON = 1, LOC_VAR = 2;

__device__ __forceinline__ double clamp4(double x) { return x > 1e4 ? 1e4 : (x < 1e-4 ? 1e-4 : x); }

// _soc_block_scale_value_scalar (scaling.jl:245-473)
__device__ double block_value(int64_t len, double bmax, double rms, int st, int ph, int loc, int64_t count) {
  const int64_t AD = 8, PR = 512, MANY = 100000;
  if (len <= 0) return 1.0;
  double geo = sqrt(bmax * rms);
  switch (st) {
    case HPR_SOC_SCALE_MAX: return bmax;
    case HPR_SOC_SCALE_RMS: return rms;
    case HPR_SOC_SCALE_GEOM: return geo;
    case HPR_SOC_SCALE_ADAPTIVE: return len <= AD ? bmax : rms;
    case HPR_SOC_SCALE_HYBRID:
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_POCK) return rms;
      return geo;
    case HPR_SOC_SCALE_RUIZ_GEOM:
      if (ph == PH_RUIZ) return len <= AD ? bmax : geo;
      if (ph == PH_POCK) return rms;
      return geo;
    case HPR_SOC_SCALE_ROLE_SPLIT:
      if (loc == LOC_CON) return geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_POCK) return rms;
      return geo;
    case HPR_SOC_SCALE_POCK_SAFE_ROLE_SPLIT:
      if (ph == PH_POCK) return bmax;
      if (loc == LOC_CON) return geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      return geo;
    case HPR_SOC_SCALE_SIZE_SPLIT_ROLE_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_POCK) return len <= PR ? rms : bmax;
      return geo;
    case HPR_SOC_SCALE_PRE_POCK_SIZE_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= PR ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo;
    case HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER:
    case HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER_POCK_GEOM: {
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= PR ? rms : sqrt(sqrt(bmax * (rms * rms * rms)));
      if (ph == PH_POCK) {
        if (st == HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER) return bmax;
        return len <= PR ? bmax : geo;
      }
      return geo;
    }
    case HPR_SOC_SCALE_PRE_POCK_BAND_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo;
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= AD ? bmax : (len <= PR ? rms : bmax);
      if (ph == PH_POCK) return bmax;
      return geo;
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS:
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX:
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER:
    case HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX:
    case HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS: {
      if (loc == LOC_CON) {
        if (ph == PH_POCK) return bmax;
        if (st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS && ph == PH_PRE_POCK) return rms;
        if (st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX && ph == PH_PRE_POCK) return bmax;
        if (st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER && ph == PH_PRE_POCK)
          return sqrt(sqrt(bmax * (rms * rms * rms)));
        if (st == HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX && (ph == PH_RUIZ || ph == PH_PRE_POCK))
          return len <= AD ? bmax : geo;
        if (st == HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS && count >= MANY && len <= AD) {
          if (ph == PH_RUIZ) return sqrt(sqrt((bmax * bmax * bmax) * rms));
          if (ph == PH_PRE_POCK) return bmax;
        }
        return geo;
      }
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= PR ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo;
    }
    case HPR_SOC_SCALE_PHASE_BLEND:
    case HPR_SOC_SCALE_PHASE_TAPER:
      if (ph == PH_RUIZ) return len <= AD ? bmax : rms;
      if (ph == PH_POCK) return len <= AD ? rms : geo;
      return geo;
  }
  return bmax;
}

bool uses_pre_pock(int st) {
  return st == HPR_SOC_SCALE_PRE_POCK_SIZE_SPLIT || st == HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER ||
         st == HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER_POCK_GEOM || st == HPR_SOC_SCALE_PRE_POCK_BAND_SPLIT ||
         st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS || st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX ||
         st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER || st == HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX ||
         st == HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS;
}

// The three kernels below give each row (or cone) a group of G lanes that
// walk its entries with stride G, so a warp's loads are coalesced and a long
// row or cone is spread over G lanes instead of one thread (G = 1: one
// thread per row, entries in order).  G is chosen per launch from the mean
// length.  Maxima do not depend on the order; sums are added per lane and
// then over the group in a fixed shuffle order, so the result depends on
// the data and G only.
template <int G>
__device__ __forceinline__ double group_combine(double v, bool sum) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) {
    const double o = __shfl_down_sync(0xffffffffu, v, off, G);
    if (((threadIdx.x & 31) % G) + off < G) v = sum ? v + o : cmax(v, o);
  }
  return v;
}

// compute_row_max_abs(_with_Q)_kernel! / compute_row_sum_abs_kernel! /
// compute_col_sum_abs_with_Q_kernel! (kernels.jl:6699-6798, 6965-7030)
template <int G>
__global__ void row_stat_kernel(int64_t nr, const int32_t* rp, const double* v, const int32_t* qrp,
                                const double* qv, int use_sum, double* out) {
  constexpr int kRows = 32 / G;  // rows per warp step
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b0 = w * kRows; b0 < nr; b0 += nw * kRows) {
    const int64_t i = b0 + lane / G;
    double q = 0.0, a = 0.0;
    if (i < nr) {
      if (qrp)
        for (int64_t k = qrp[i] + sub; k < qrp[i + 1]; k += G) q = use_sum ? q + fabs(qv[k]) : cmax(q, fabs(qv[k]));
      for (int64_t k = rp[i] + sub; k < rp[i + 1]; k += G) a = use_sum ? a + fabs(v[k]) : cmax(a, fabs(v[k]));
    }
    q = group_combine<G>(q, use_sum != 0);
    a = group_combine<G>(a, use_sum != 0);
    if (i < nr && sub == 0) {
      const double r = use_sum ? q + a : cmax(q, a);
      out[i] = clamp4(r > 0.0 ? sqrt(r) : 1.0);
    }
  }
}

// apply_soc_block_scaling(_phase_taper)_kernel! (kernels.jl:6820-6920)
template <int G>
__global__ void block_kernel(int64_t ncones, const int32_t* cs, double* t, int st, int ph, int loc) {
  constexpr int kCones = 32 / G;
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b0 = w * kCones; b0 < ncones; b0 += nw * kCones) {
    const int64_t k = b0 + lane / G;
    int64_t a = 0, b = 0;
    if (k < ncones) {
      a = cs[k];
      b = cs[k + 1];
    }
    double bmax = 0.0, ss = 0.0;
    for (int64_t j = a + sub; j < b; j += G) {
      bmax = cmax(bmax, t[j]);
      ss = fma(t[j], t[j], ss);
    }
    // every lane of the group has read its entries before any is written
    bmax = group_combine<G>(bmax, false);
    ss = group_combine<G>(ss, true);
    bmax = __shfl_sync(0xffffffffu, bmax, lane - sub);
    ss = __shfl_sync(0xffffffffu, ss, lane - sub);
    const int64_t len = b - a;
    if (len <= 0) continue;
    const double rms = st == HPR_SOC_SCALE_MAX ? bmax : sqrt(ss / (double)len);
    const double val = block_value(len, bmax, rms, st, ph, loc, ncones);
    for (int64_t j = a + sub; j < b; j += G) t[j] = val;
  }
}

// scale_csr_row_col_kernel! (kernels.jl:7120-7140)
template <int G>
__global__ void scale_csr_kernel(int64_t nr, const int32_t* rp, const int32_t* ci, double* v, const double* r,
                                 const double* cl) {
  constexpr int kRows = 32 / G;
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b0 = w * kRows; b0 < nr; b0 += nw * kRows) {
    const int64_t i = b0 + lane / G;
    if (i >= nr) continue;
    const double rinv = 1.0 / r[i];
    for (int64_t k = rp[i] + sub; k < rp[i + 1]; k += G) {
      double x = v[k];
      x *= rinv;
      x /= cl[ci[k]];
      v[k] = x;
    }
  }
}

// check_diagonal_kernel! / extract_diagonal_csr_kernel! (kernels.jl:7034-7084)
struct DiagCheckF {
  const int32_t *rp, *ci;
  const double* v;
  double* dq;
  __device__ void operator()(int64_t i, Red& r) const {
    int64_t a = rp[i], b = rp[i + 1];
    double isd = 1.0;
    if (b - a == 1) isd = (ci[a] == i) ? 1.0 : 0.0;
    else if (b - a > 1) isd = 0.0;
    double d = 0.0, rs = 0.0;
    for (int64_t k = a; k < b; ++k) {
      rs += fabs(v[k]);
      if (ci[k] == i && d == 0.0) d = v[k];
    }
    dq[i] = d;
    r.v[0] = r.v[0] + (1.0 - isd);           // rows that are not diagonal
    r.v[1] = nanmax(r.v[1], fabs(rs - fabs(d)));
  }
};

// ||max(|AL_fin|, |AU_fin|)||_{inf,2}, ||soc_rhs||_inf, ||c||_{inf,2}
struct BNormF {
  const double *al, *au;
  __device__ void operator()(int64_t i, Red& r) const {
    double a = (al[i] == -INFINITY) ? 0.0 : al[i];
    double b = (au[i] == INFINITY) ? 0.0 : au[i];
    double v = cmax(fabs(a), fabs(b));
    r.v[0] = nanmax(r.v[0], v);
    r.v[1] = r.v[1] + v * v;
  }
};
struct VNormF {
  const double* a;
  __device__ void operator()(int64_t i, Red& r) const {
    r.v[0] = nanmax(r.v[0], fabs(a[i]));
    r.v[1] = r.v[1] + a[i] * a[i];
  }
};
struct FinF {
  const double* a;
  __device__ void operator()(int64_t i, Red& r) const {
    double x = a[i];
    if (isfinite(x)) {
      r.v[0] = nanmax(r.v[0], fabs(x));
      r.v[1] = fma(x, x, r.v[1]);
      r.v[2] = r.v[2] + 1.0;
    }
  }
};

int bnorms(Ctx* c, double* inf_, double* l2_) {
  const int64_t m = c->m, n = c->n;
  const int64_t ncon = (int64_t)c->h_con_idx.size() - 1;
  const int64_t nrhs = m - c->m_lin;
  const bool have_rhs = ncon > 0 && nrhs > 0;
  if (m > 0) HPR_TRY(vec_reduce<2, 1>(c, m, BNormF{c->AL, c->AU}, 0));
  else HPR_CUDA(c, cudaMemsetAsync(c->d_red_out, 0, 2 * sizeof(double), c->stream));
  HPR_TRY(vec_reduce<2, 1>(c, have_rhs ? nrhs : 0, VNormF{c->soc_rhs}, 2));
  HPR_TRY(vec_reduce<2, 1>(c, n, VNormF{c->c}, 4));
  HPR_TRY(fetch_red(c, 6));
  const double* h = c->h_red_out;
  inf_[0] = h[0];
  l2_[0] = std::sqrt(h[1]);
  inf_[1] = have_rhs ? h[2] : 0.0;
  l2_[1] = have_rhs ? std::sqrt(h[3]) : 0.0;
  inf_[2] = h[4];
  l2_[2] = std::sqrt(h[5]);
  return HPR_OK;
}

inline int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// lanes per row (or cone) for a mean length of `mean` entries
inline int group_lanes(double mean) { return mean <= 6.0 ? 4 : (mean <= 12.0 ? 8 : (mean <= 24.0 ? 16 : 32)); }

template <int G>
void row_stat_g(Ctx* c, int64_t nr, const int32_t* rp, const double* v, const int32_t* qrp, const double* qv,
                int use_sum, double* out) {
  row_stat_kernel<G><<<grid_for(nr * G), 256, 0, c->stream>>>(nr, rp, v, qrp, qv, use_sum, out);
}
// Row statistics keep one thread per row (each thread's loads run ahead
// along its row) unless rows are long on average; measured on B200 for the
// benchmark's A and A' (means 17 and 12): 150 / 50 us per pass with one
// thread per row against 388 / 300 us with 16 lanes per row.
void row_stat(Ctx* c, int64_t nr, int64_t nnz, const int32_t* rp, const double* v, const int32_t* qrp,
              const double* qv, int use_sum, double* out) {
  if ((double)nnz / (double)std::max<int64_t>(nr, 1) <= 64.0) row_stat_g<1>(c, nr, rp, v, qrp, qv, use_sum, out);
  else row_stat_g<32>(c, nr, rp, v, qrp, qv, use_sum, out);
}
void block_scale(Ctx* c, int64_t ncones, int64_t len, const int32_t* cs, double* t, int st, int ph, int loc) {
  const int g = group_lanes((double)len / (double)std::max<int64_t>(ncones, 1));
  const int grid = grid_for(ncones * g);
  switch (g) {
    case 4: block_kernel<4><<<grid, 256, 0, c->stream>>>(ncones, cs, t, st, ph, loc); break;
    case 8: block_kernel<8><<<grid, 256, 0, c->stream>>>(ncones, cs, t, st, ph, loc); break;
    case 16: block_kernel<16><<<grid, 256, 0, c->stream>>>(ncones, cs, t, st, ph, loc); break;
    default: block_kernel<32><<<grid, 256, 0, c->stream>>>(ncones, cs, t, st, ph, loc); break;
  }
}
void scale_csr(Ctx* c, const DevCSR& M, const double* r, const double* cl) {
  const int64_t nr = M.nrows;
  if (nr == 0) return;
  // two to four entries per lane on average
  const double mean = (double)M.nnz / (double)nr;
  const int g = mean < 16.0 ? 4 : (mean < 32.0 ? 8 : (mean < 64.0 ? 16 : 32));
  const int grid = grid_for(nr * g);
  switch (g) {
    case 4: scale_csr_kernel<4><<<grid, 256, 0, c->stream>>>(nr, M.rowptr, M.col, M.val, r, cl); break;
    case 8: scale_csr_kernel<8><<<grid, 256, 0, c->stream>>>(nr, M.rowptr, M.col, M.val, r, cl); break;
    case 16: scale_csr_kernel<16><<<grid, 256, 0, c->stream>>>(nr, M.rowptr, M.col, M.val, r, cl); break;
    default: scale_csr_kernel<32><<<grid, 256, 0, c->stream>>>(nr, M.rowptr, M.col, M.val, r, cl); break;
  }
}

int scale_pass(Ctx* c, int st, int phase, int use_sum) {
  const int64_t m = c->m, n = c->n;
  const int64_t ncon = (int64_t)c->h_con_idx.size() - 1;
  const int64_t nvar = (int64_t)c->h_var_idx.size() - 1;
  double *tr = c->vtmp_m, *tc = c->vtmp_n;
  const bool hq = c->q_kind == HPR_Q_CSR;

      row_stat(c, n, c->AT.nnz + (hq ? c->Q.nnz : 0), c->AT.rowptr, c->AT.val, hq ? c->Q.rowptr : nullptr,
               hq ? c->Q.val : nullptr, use_sum, tc);
      if (m > 0) {
        row_stat(c, m, c->A.nnz, c->A.rowptr, c->A.val, nullptr, nullptr, use_sum, tr);
        if (ncon > 0) block_scale(c, ncon, m - c->m_lin, c->d_con_start, tr, st, phase, LOC_CON);
        HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { tr[i] = clamp4(tr[i]); }));
      }
      if (nvar > 0) block_scale(c, nvar, n - c->n_box, c->d_var_start, tc, st, phase, LOC_VAR);
      HPR_CUDA(c, cudaGetLastError());
      HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { tc[i] = clamp4(tc[i]); }));
      double *rn = c->row_norm, *cn = c->col_norm;
      HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { rn[i] *= tr[i]; }));
      HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { cn[i] *= tc[i]; }));
      if (hq) scale_csr(c, c->Q, tc, tc);
      if (m > 0) {
        scale_csr(c, c->A, tr, tc);
        scale_csr(c, c->AT, tc, tr);
      }
      HPR_CUDA(c, cudaGetLastError());
      double *cc = c->c, *al = c->AL, *au = c->AU, *rh = c->soc_rhs, *rf = c->soc_rhs_full, *l = c->l, *u = c->u;
      const int64_t ml = c->m_lin;
      HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) {
        cc[i] /= tc[i];
        l[i] *= tc[i];
        u[i] *= tc[i];
      }));
      if (m > 0) {
        HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) {
          double f = tr[i];
          al[i] /= f;
          au[i] /= f;
          rf[i] /= f;
          if (i >= ml) rh[i - ml] /= f;
        }));
      }
      return HPR_OK;
    }

}  // namespace

int run_scaling(Ctx* c, const hpr_params* p, hpr_scale_info* out) {
  const int64_t m = c->m, n = c->n;
  const int64_t ncon = (int64_t)c->h_con_idx.size() - 1;
  const int64_t nvar = (int64_t)c->h_var_idx.size() - 1;
  const double *AL = c->AL, *AU = c->AU, *rhs = c->soc_rhs, *cv = c->c;
  const int64_t nrhs = m - c->m_lin;
  const bool have_rhs = ncon > 0 && nrhs > 0;
  double ninf[3], nl2[3];
  HPR_TRY(bnorms(c, ninf, nl2));
  auto jmax = [](double a, double b) { return std::max(a, b); };
  c->norm_b_org = m > 0 ? jmax(ninf[0], ninf[1]) : 0.0;
  c->norm_c_org = ninf[2];

  // row_norm = col_norm = 1
  {
    double *rn = c->row_norm, *cn = c->col_norm;
    HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { rn[i] = 1.0; }));
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { cn[i] = 1.0; }));
  }
  if (c->q_kind == HPR_Q_DIAG_LOWRANK || c->q_kind == HPR_Q_OPERATOR) {
    // operator Q: no scaling at all (scaling.jl:800-846)
    c->b_scale = c->c_scale = 1.0;
    c->norm_b = m > 0 ? jmax(nl2[0], ninf[1]) : 0.0;
    c->norm_c = nl2[2];
  } else {
    const bool hq = c->q_kind == HPR_Q_CSR;
    const int st = p->soc_block_scaling_strategy;
    if (p->use_Ruiz_scaling)
      for (int it = 0; it < std::max(p->ruiz_iterations, 0); ++it) HPR_TRY(scale_pass(c, st, PH_RUIZ, 0));
    if (uses_pre_pock(st))
      for (int it = 0; it < 2; ++it) HPR_TRY(scale_pass(c, st, PH_PRE_POCK, 0));
    if (p->use_Pock_Chambolle_scaling) HPR_TRY(scale_pass(c, st, PH_POCK, 1));
    if (p->use_bc_scaling) {
      // compute_bc_scales (scaling.jl:722-729)
      const int nt = p->bc_scaling_norm_type;
      HPR_TRY(vec_reduce<3, 1>(c, m, FinF{AL}, 0));
      HPR_TRY(vec_reduce<3, 1>(c, m, FinF{AU}, 3));
      HPR_TRY(vec_reduce<2, 1>(c, have_rhs ? nrhs : 0, VNormF{rhs}, 6));
      HPR_TRY(vec_reduce<2, 1>(c, n, VNormF{cv}, 8));
      HPR_TRY(fetch_red(c, 10));
      const double* h = c->h_red_out;
      auto fin = [&](const double* r) {
        if (nt == HPR_BC_NORM_LINF) return r[0];
        if (r[2] == 0.0) return 0.0;
        return nt == HPR_BC_NORM_RMS ? std::sqrt(r[1] / r[2]) : std::sqrt(r[1]);
      };
      auto vnorm = [&](const double* r, int64_t len) {
        if (len <= 0) return 0.0;
        if (nt == HPR_BC_NORM_LINF) return r[0];
        return nt == HPR_BC_NORM_RMS ? std::sqrt(r[1] / (double)len) : std::sqrt(r[1]);
      };
      auto clip = [](double x) { return std::min(std::max(x, 1e-4), 1e4); };
      double srhs = have_rhs ? vnorm(h + 6, nrhs) : 0.0;
      double hb = clip(std::max({1.0, fin(h + 0), fin(h + 3), srhs}));
      double hc = clip(std::max(1.0, vnorm(h + 8, n)));
      double sb = hb;
      double sc = hc > hb / 1e-2 ? hb / 1e-2 : (hc < hb / 1e2 ? hb / 1e2 : hc);
      if (hq && c->Q.nnz > 0) {
        double f = sb / sc;
        double* qv = c->Q.val;
        HPR_TRY(vec_map(c, c->Q.nnz, [=] __device__(int64_t k) { qv[k] *= f; }));
      }
      double *al = c->AL, *au = c->AU, *rh = c->soc_rhs, *rf = c->soc_rhs_full, *cc = c->c, *l = c->l, *u = c->u;
      const int64_t ml = c->m_lin;
      if (m > 0)
        HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) {
          al[i] /= sb;
          au[i] /= sb;
          rf[i] /= sb;
          if (i >= ml) rh[i - ml] /= sb;
        }));
      HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) {
        cc[i] /= sc;
        l[i] /= sb;
        u[i] /= sb;
      }));
      c->b_scale = sb;
      c->c_scale = sc;
    } else {
      c->b_scale = c->c_scale = 1.0;
    }
    HPR_TRY(bnorms(c, ninf, nl2));
    c->norm_b = jmax(nl2[0], ninf[1]);
    c->norm_c = nl2[2];
  }
  // check_Q_diagonal (GPU form, scaling.jl:1327-1353)
  if (c->q_kind == HPR_Q_CSR) {
    HPR_TRY(vec_reduce<2, 2>(c, n, DiagCheckF{c->Q.rowptr, c->Q.col, c->Q.val, c->diag_Q}, 0));
    HPR_TRY(fetch_red(c, 2));
    c->Q_is_diag = (c->h_red_out[0] == 0.0) && (c->h_red_out[1] <= 1e-10);
  } else if (c->q_kind == HPR_Q_NONE) {
    HPR_CUDA(c, cudaMemsetAsync(c->diag_Q, 0, std::max<int64_t>(n, 1) * sizeof(double), c->stream));
    c->Q_is_diag = true;
  } else {
    c->Q_is_diag = false;
  }
  // the matrices' values changed: the engine's tiled copies are rebuilt
  for (DevCSR* M : {&c->A, &c->AT, &c->Q, &c->F, &c->FT}) ++M->version;
  HPR_TRY(prepare_engine(c));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  c->scaled = true;
  if (out) {
    out->b_scale = c->b_scale;
    out->c_scale = c->c_scale;
    out->norm_b = c->norm_b;
    out->norm_c = c->norm_c;
    out->norm_b_org = c->norm_b_org;
    out->norm_c_org = c->norm_c_org;
    out->Q_is_diag = c->Q_is_diag ? 1 : 0;
  }
  return HPR_OK;
}

}  // namespace hpr
