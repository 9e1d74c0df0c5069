// hpr_oracle.cpp — CPU FP64 restatement of the reference HPR-SOCP solver.
//
// TEST INFRASTRUCTURE ONLY (see hpr_oracle.h).  Every routine below follows a
// reference function (PolyU-IOR/HPR-SOCP, Julia) cited beside it.  Arithmetic
// follows the reference's operation order: `muladd` in the reference becomes
// std::fma here (this file is compiled with -ffp-contract=off so nothing else
// is fused), and sparse matrix-vector products sum each output element in
// ascending column order with separately rounded multiply and add, which is
// what Julia's SparseMatrixCSC `mul!` does.
//
// Where the reference's CPU and GPU paths differ only in rounding order the
// GPU form is used, because the GPU is the reference's production path:
//   * scaling clamps the sqrt'ed norms to [1e-4, 1e4] inside the norm pass
//     and again after SOC block aggregation (kernels.jl:6699-6798, 7034-7148);
//   * A and A' are scaled separately as v*(1/r_i)/c_j (kernels.jl:7120-7140);
//   * Q is not re-symmetrised after scaling (scaling.jl:1264-1268 is CPU only).
#include "hpr_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

using std::vector;

namespace {

// Persistent worker pool (the image has no OpenMP runtime).  par_for splits
// [lo, hi) into chunks of `grain` and runs them on all workers plus the
// caller; results never depend on the thread count.
class Pool {
 public:
  void resize(int n) {
    stop();
    nthreads_ = std::max(1, n);
    quit_ = false;
    for (int t = 1; t < nthreads_; ++t) workers_.emplace_back([this] { loop(); });
  }
  int size() const { return nthreads_; }
  void run(int64_t nchunks, const std::function<void(int64_t)>& job) {
    if (nthreads_ <= 1 || nchunks <= 1) {
      for (int64_t k = 0; k < nchunks; ++k) job(k);
      return;
    }
    {
      std::unique_lock<std::mutex> lk(mu_);
      job_ = &job;
      nchunks_ = nchunks;
      next_.store(0);
      active_ = nthreads_ - 1;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return active_ == 0; });
    job_ = nullptr;
  }
  ~Pool() { stop(); }

 private:
  void work() {
    for (;;) {
      int64_t k = next_.fetch_add(1);
      if (k >= nchunks_) break;
      (*job_)(k);
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_;
      }
      work();
      std::unique_lock<std::mutex> lk(mu_);
      if (--active_ == 0) done_cv_.notify_one();
    }
  }
  void stop() {
    {
      std::unique_lock<std::mutex> lk(mu_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    workers_.clear();
  }
  int nthreads_ = 1;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int64_t)>* job_ = nullptr;
  int64_t nchunks_ = 0;
  std::atomic<int64_t> next_{0};
  int active_ = 0;
  uint64_t gen_ = 0;
  bool quit_ = false;
};
Pool g_pool;

template <class F>
void par_for(int64_t lo, int64_t hi, F f, int64_t grain) {
  if (hi <= lo) return;
  int64_t n = hi - lo;
  if (g_pool.size() <= 1 || n <= grain) {
    for (int64_t i = lo; i < hi; ++i) f(i);
    return;
  }
  int64_t nchunks = (n + grain - 1) / grain;
  std::function<void(int64_t)> job = [&](int64_t k) {
    int64_t b = lo + k * grain, e = std::min(hi, b + grain);
    for (int64_t i = b; i < e; ++i) f(i);
  };
  g_pool.run(nchunks, job);
}

const double INF = std::numeric_limits<double>::infinity();

struct CSR {
  int64_t nr = 0, nc = 0;
  vector<int64_t> rp;  // nr+1
  vector<int32_t> ci;
  vector<double> v;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

CSR transpose(const CSR& A) {
  CSR T;
  T.nr = A.nc;
  T.nc = A.nr;
  T.rp.assign(T.nr + 1, 0);
  for (int64_t k = 0; k < A.nnz(); ++k) T.rp[A.ci[k] + 1]++;
  for (int64_t i = 0; i < T.nr; ++i) T.rp[i + 1] += T.rp[i];
  T.ci.resize(A.nnz());
  T.v.resize(A.nnz());
  vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t i = 0; i < A.nr; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int64_t p = pos[A.ci[k]]++;
      T.ci[p] = (int32_t)i;
      T.v[p] = A.v[k];
    }
  return T;
}

// y = A x, one sequential sum per row in ascending column order.
void spmv(const CSR& A, const double* x, double* y) {
  par_for(0, A.nr, [&](int64_t i) {
    double s = 0.0;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      double p = A.v[k] * x[A.ci[k]];
      s = s + p;
    }
    y[i] = s;
  }, 1024);
}

// Deterministic sums: fixed 4096-element blocks summed sequentially, then the
// block sums in order, independent of the thread count.
const int64_t RBLK = 4096;
template <class F>
double det_sum(int64_t n, F f) {
  if (n <= 0) return 0.0;
  int64_t nb = (n + RBLK - 1) / RBLK;
  vector<double> part(nb);
  par_for(0, nb, [&](int64_t b) {
    double s = 0.0;
    int64_t e = std::min(n, (b + 1) * RBLK);
    for (int64_t i = b * RBLK; i < e; ++i) s += f(i);
    part[b] = s;
  }, 1);
  double s = 0.0;
  for (int64_t b = 0; b < nb; ++b) s += part[b];
  return s;
}
double dot(const vector<double>& a, const vector<double>& b) {
  const double* pa = a.data();
  const double* pb = b.data();
  return det_sum((int64_t)a.size(), [&](int64_t i) { return pa[i] * pb[i]; });
}
double nrm2(const vector<double>& a) { return std::sqrt(dot(a, a)); }
// Julia maximum(abs, x): NaN propagates.
inline double jmax(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return a > b ? a : b;
}
inline double jmin(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return a < b ? a : b;
}
double absmax_range(const double* x, int64_t lo, int64_t hi) {
  if (hi <= lo) return 0.0;
  int64_t nb = (hi - lo + RBLK - 1) / RBLK;
  vector<double> part(nb, 0.0);
  par_for(0, nb, [&](int64_t b) {
    double m = 0.0;
    int64_t e = std::min(hi, lo + (b + 1) * RBLK);
    for (int64_t i = lo + b * RBLK; i < e; ++i) m = jmax(m, std::fabs(x[i]));
    part[b] = m;
  }, 1);
  double m = 0.0;
  for (double v : part) m = jmax(m, v);
  return m;
}
double absmax(const vector<double>& x) {
  return absmax_range(x.data(), 0, (int64_t)x.size());
}
// Julia clamp(x, lo, hi) = ifelse(x > hi, hi, ifelse(x < lo, lo, x))
inline double jclamp(double x, double lo, double hi) {
  return x > hi ? hi : (x < lo ? lo : x);
}

// Start vector of the power iteration.  The reference draws
// randn(MersenneTwister(1)) .+ 1e-8 (eigenvalues.jl:72-76), which cannot be
// reproduced outside Julia; both this oracle and the CUDA library use the same
// splitmix64 uniform(-1,1) vector plus 1e-8 instead.
void start_vector(vector<double>& z, uint64_t seed) {
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

}  // namespace

struct oracle_ctx {
  std::string err;
  int threads = 0;
  // ---- problem (canonical, 0-based), QP_info_cpu (structs.jl:97-150)
  int64_t m = 0, n = 0, m_lin = 0, n_box = 0;
  CSR A, AT;
  vector<double> c, l, u, AL, AU, soc_rhs, soc_rhs_full;
  vector<int64_t> con_idx, var_idx;  // starts + end sentinel, 0-based
  int q_kind = HPR_Q_NONE;
  CSR Q, F, FT;
  vector<double> qdiag;  // operator D
  double obj_constant = 0.0;
  bool has_q = false;
  // ---- scaling (Scaling_info_cpu, structs.jl:153-166)
  vector<double> row_norm, col_norm, l_org, u_org, soc_con_scale,
      soc_var_scale;
  double b_scale = 1, c_scale = 1, norm_b = 0, norm_c = 0, norm_b_org = 0,
         norm_c_org = 0;
  bool scaled = false;
  bool Q_is_diag = false;
  vector<double> diag_Q;
  // ---- workspace (HPRSOCP_workspace_cpu, structs.jl:529-597)
  vector<double> w, w_bar, dw, x, x_hat, x_bar, dx, y, y_bar, dy, z_bar, Rp,
      Rd, Ax, ATy, ATy_bar, ATdy, QATdy, s, Qw, Qw_bar, Qx, dQw, last_x, last_y,
      last_w, last_ATy, tempv, fact1, fact2, fact, fact_M, ftmp;
  double sigma = 1.0, lamA = 0.0, lamQ = 0.0;
  int64_t inner = 0;
  bool to_check = true;

  int64_t ncon() const { return (int64_t)con_idx.size() - 1; }
  int64_t nvar() const { return (int64_t)var_idx.size() - 1; }
  int64_t linear_n() const { return nvar() > 0 ? n_box : n; }

  // Qmap! (sparse_matrix_operator.jl:27-51, Q_operator_interface.jl:32-34)
  void qmap(const vector<double>& v, vector<double>& out) {
    if (q_kind == HPR_Q_CSR) {
      spmv(Q, v.data(), out.data());
    } else if (q_kind == HPR_Q_DIAG_LOWRANK) {
      spmv(F, v.data(), ftmp.data());
      const double* t = ftmp.data();
      par_for(0, n, [&](int64_t i) {
        double s = 0.0;
        for (int64_t k = FT.rp[i]; k < FT.rp[i + 1]; ++k) {
          double p = FT.v[k] * t[FT.ci[k]];
          s = s + p;
        }
        out[i] = qdiag[i] * v[i] + s;
      }, 1024);
    } else {
      std::fill(out.begin(), out.end(), 0.0);
    }
  }
};

static int fail(oracle_ctx* o, int code, const std::string& msg) {
  if (o) o->err = msg;
  return code;
}

static bool load_csr(const hpr_csr& s, int base, CSR& d, std::string& err,
                     const char* name) {
  d.nr = s.nrows;
  d.nc = s.ncols;
  d.rp.resize(d.nr + 1);
  d.ci.resize(s.nnz);
  d.v.resize(s.nnz);
  if (d.nr > 0 && !s.rowptr) {
    err = std::string(name) + ": null rowptr";
    return false;
  }
  for (int64_t i = 0; i <= d.nr; ++i) d.rp[i] = (d.nr > 0) ? s.rowptr[i] - base : 0;
  if (d.rp[0] != 0 || d.rp[d.nr] != s.nnz) {
    err = std::string(name) + ": rowptr does not span nnz";
    return false;
  }
  for (int64_t k = 0; k < s.nnz; ++k) {
    d.ci[k] = s.colind[k] - base;
    d.v[k] = s.values[k];
    if (d.ci[k] < 0 || d.ci[k] >= d.nc) {
      err = std::string(name) + ": column index out of range";
      return false;
    }
  }
  return true;
}

extern "C" {

void oracle_default_params(hpr_params* p) {
  // HPRSOCP_parameters() defaults (structs.jl:277)
  std::memset(p, 0, sizeof(*p));
  p->stoptol = 1e-6;
  p->sigma = -1;
  p->max_iter = 2147483647;
  p->time_limit = 3600.0;
  p->check_iter = 150;
  p->print_frequency = -1;
  p->device_number = 0;
  p->use_Ruiz_scaling = 1;
  p->ruiz_iterations = 10;
  p->use_bc_scaling = 1;
  p->bc_scaling_norm_type = HPR_BC_NORM_L2;
  p->use_Pock_Chambolle_scaling = 1;
  p->soc_block_scaling_strategy = HPR_SOC_SCALE_PHASE_TAPER;
  p->verbose = 0;
  p->lambda_max_A = -1;
  p->lambda_max_Q = -1;
  p->precision = HPR_PREC_FP64;
  p->refine = 0;
}

const char* oracle_last_error(const oracle_ctx* o) {
  return o ? o->err.c_str() : "null context";
}

// build_from_SOCP_data layout (builders.jl:24-108), taken as given.
int oracle_create(const hpr_problem* p, int threads, oracle_ctx** out) {
  *out = nullptr;
  oracle_ctx* o = new oracle_ctx();
  o->threads = threads;
  {
    int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
    if (nt != g_pool.size()) g_pool.resize(nt);
  }
  int base = p->index_base;
  o->m = p->m;
  o->n = p->n;
  o->m_lin = p->m_lin;
  o->n_box = p->n_box;
  std::string err;
  if (p->A.nrows != p->m || p->A.ncols != p->n) {
    delete o;
    return HPR_E_BAD_INPUT;
  }
  if (!load_csr(p->A, base, o->A, err, "A")) {
    delete o;
    return HPR_E_BAD_INPUT;
  }
  if (p->AT.rowptr) {
    if (!load_csr(p->AT, base, o->AT, err, "AT")) {
      delete o;
      return HPR_E_BAD_INPUT;
    }
  } else {
    o->AT = transpose(o->A);
  }
  int64_t m = o->m, n = o->n;
  o->c.assign(p->c, p->c + n);
  o->l.assign(p->l, p->l + n);
  o->u.assign(p->u, p->u + n);
  o->AL.assign(p->AL, p->AL + m);
  o->AU.assign(p->AU, p->AU + m);
  o->soc_rhs.assign(m - o->m_lin, 0.0);
  if (p->soc_rhs)
    for (int64_t i = 0; i < m - o->m_lin; ++i) o->soc_rhs[i] = p->soc_rhs[i];
  o->soc_rhs_full.assign(m, 0.0);
  for (int64_t i = o->m_lin; i < m; ++i) o->soc_rhs_full[i] = o->soc_rhs[i - o->m_lin];
  for (int64_t k = 0; k < p->n_soc_con_idx; ++k) o->con_idx.push_back(p->soc_con_idx[k] - base);
  for (int64_t k = 0; k < p->n_soc_var_idx; ++k) o->var_idx.push_back(p->soc_var_idx[k] - base);
  if (o->con_idx.empty()) o->con_idx.push_back(m);
  if (o->var_idx.empty()) o->var_idx.push_back(n);
  o->q_kind = p->q_kind;
  if (p->q_kind == HPR_Q_CSR) {
    if (!load_csr(p->Q, base, o->Q, err, "Q")) {
      delete o;
      return HPR_E_BAD_INPUT;
    }
    o->has_q = o->Q.nnz() > 0;  // has_quadratic_terms (Q_operator_interface.jl:118-121)
    if (!o->has_q) o->q_kind = HPR_Q_NONE;
  } else if (p->q_kind == HPR_Q_DIAG_LOWRANK) {
    if (!load_csr(p->F, base, o->F, err, "F")) {
      delete o;
      return HPR_E_BAD_INPUT;
    }
    o->FT = transpose(o->F);
    o->qdiag.assign(p->q_diag, p->q_diag + n);
    o->ftmp.assign(o->F.nr, 0.0);
    o->has_q = true;  // operators always count as quadratic
  }
  o->obj_constant = p->obj_constant;
  // workspace (allocate_workspace, algorithm.jl:1443-1588)
  for (auto* v : {&o->w, &o->w_bar, &o->dw, &o->x, &o->x_hat, &o->x_bar, &o->dx,
                  &o->z_bar, &o->Rd, &o->ATy, &o->ATy_bar, &o->ATdy, &o->QATdy,
                  &o->Qw, &o->Qw_bar, &o->Qx, &o->dQw, &o->last_x, &o->last_w,
                  &o->last_ATy, &o->tempv, &o->fact1, &o->fact2, &o->fact,
                  &o->fact_M})
    v->assign(n, 0.0);
  for (auto* v : {&o->y, &o->y_bar, &o->dy, &o->Rp, &o->Ax, &o->s, &o->last_y})
    v->assign(m, 0.0);
  o->row_norm.assign(m, 1.0);
  o->col_norm.assign(n, 1.0);
  o->l_org = o->l;
  o->u_org = o->u;
  o->soc_con_scale.assign(std::max<int64_t>(o->ncon(), 0), 1.0);
  o->soc_var_scale.assign(std::max<int64_t>(o->nvar(), 0), 1.0);
  o->diag_Q.assign(n, 0.0);
  // norms of the unscaled data, as an unscaled solve would report them
  *out = o;
  return HPR_OK;
}

void oracle_destroy(oracle_ctx* o) { delete o; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Scaling (scaling!, scaling.jl:785-1289)
// ---------------------------------------------------------------------------
namespace {

const int PH_GENERIC = 0, PH_RUIZ = 1, PH_PRE_POCK = 2, PH_POCK = 3;
const int LOC_GENERIC = 0, LOC_CON = 1, LOC_VAR = 2;
const int64_t ADAPT = 8, POCK_RMS = 512, MANY_CON = 100000;

// _soc_block_scale_value_scalar (scaling.jl:245-473)
double block_scale_value(int64_t len, double bmax, double rms, int st, int ph,
                         int loc, int64_t cone_count) {
  if (len <= 0) return 1.0;
  if (st == HPR_SOC_SCALE_MAX) return bmax;
  auto geo = [&] { return std::sqrt(bmax * rms); };
  auto taper = [&] { return std::sqrt(std::sqrt(bmax * (rms * rms * rms))); };
  auto maxb = [&] { return std::sqrt(std::sqrt((bmax * bmax * bmax) * rms)); };
  switch (st) {
    case HPR_SOC_SCALE_RMS: return rms;
    case HPR_SOC_SCALE_GEOM: return geo();
    case HPR_SOC_SCALE_ADAPTIVE: return len <= ADAPT ? bmax : rms;
    case HPR_SOC_SCALE_HYBRID:
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_POCK) return rms;
      return geo();
    case HPR_SOC_SCALE_RUIZ_GEOM:
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : geo();
      if (ph == PH_POCK) return rms;
      return geo();
    case HPR_SOC_SCALE_ROLE_SPLIT:
      if (loc == LOC_CON) return geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_POCK) return rms;
      return geo();
    case HPR_SOC_SCALE_POCK_SAFE_ROLE_SPLIT:
      if (ph == PH_POCK) return bmax;
      if (loc == LOC_CON) return geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      return geo();
    case HPR_SOC_SCALE_SIZE_SPLIT_ROLE_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_POCK) return len <= POCK_RMS ? rms : bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_SIZE_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : taper();
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER_POCK_GEOM:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : taper();
      if (ph == PH_POCK) return len <= POCK_RMS ? bmax : geo();
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_BAND_SPLIT:
      if (loc == LOC_CON) return ph == PH_POCK ? bmax : geo();
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK)
        return len <= ADAPT ? bmax : (len <= POCK_RMS ? rms : bmax);
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS:
      if (loc == LOC_CON) {
        if (ph == PH_POCK) return bmax;
        if (ph == PH_PRE_POCK) return rms;
        return geo();
      }
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX:
      if (loc == LOC_CON) {
        if (ph == PH_POCK || ph == PH_PRE_POCK) return bmax;
        return geo();
      }
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER:
      if (loc == LOC_CON) {
        if (ph == PH_POCK) return bmax;
        if (ph == PH_PRE_POCK) return taper();
        return geo();
      }
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX:
      if (loc == LOC_CON) {
        if (ph == PH_POCK) return bmax;
        if (ph == PH_RUIZ || ph == PH_PRE_POCK) return len <= ADAPT ? bmax : geo();
        return geo();
      }
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS:
      if (loc == LOC_CON) {
        bool many = cone_count >= MANY_CON && len <= ADAPT;
        if (ph == PH_POCK) return bmax;
        if (many) {
          if (ph == PH_RUIZ) return maxb();
          if (ph == PH_PRE_POCK) return bmax;
        }
        return geo();
      }
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_PRE_POCK) return len <= POCK_RMS ? rms : bmax;
      if (ph == PH_POCK) return bmax;
      return geo();
    case HPR_SOC_SCALE_PHASE_BLEND:
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_POCK) return len <= ADAPT ? rms : geo();
      return geo();
    case HPR_SOC_SCALE_PHASE_TAPER:
      if (ph == PH_RUIZ) return len <= ADAPT ? bmax : rms;
      if (ph == PH_POCK) return len <= ADAPT ? rms : geo();
      return geo();
  }
  return bmax;
}

bool uses_pre_pock(int st) {
  return st == HPR_SOC_SCALE_PRE_POCK_SIZE_SPLIT ||
         st == HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER ||
         st == HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER_POCK_GEOM ||
         st == HPR_SOC_SCALE_PRE_POCK_BAND_SPLIT ||
         st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS ||
         st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX ||
         st == HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER ||
         st == HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX ||
         st == HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS;
}

// apply_soc_block_scaling_kernel! (kernels.jl:6820-6862): sequential block
// max and fma sum of squares, one factor broadcast per cone.
void apply_block(vector<double>& t, const vector<int64_t>& idx, int st, int ph,
                 int loc) {
  int64_t nb = (int64_t)idx.size() - 1;
  for (int64_t i = 0; i < nb; ++i) {
    int64_t a = idx[i], b = idx[i + 1];
    int64_t len = b - a;
    if (len <= 0) continue;
    double bmax = 0.0, ss = 0.0;
    for (int64_t j = a; j < b; ++j) {
      bmax = std::max(bmax, t[j]);
      ss = std::fma(t[j], t[j], ss);
    }
    double rms = st == HPR_SOC_SCALE_MAX ? bmax : std::sqrt(ss / (double)len);
    double v = block_scale_value(len, bmax, rms, st, ph, loc, nb);
    for (int64_t j = a; j < b; ++j) t[j] = v;
  }
}
inline double clip4(double x) { return jclamp(x, 1e-4, 1e4); }

// compute_row_max_abs_kernel! / compute_row_max_abs_with_Q_kernel! /
// compute_row_sum_abs_kernel! / compute_col_sum_abs_with_Q_kernel!
// (kernels.jl:6699-6798, 6965-7030)
void row_stat(const CSR& M, const CSR* Qm, bool use_sum, vector<double>& outv) {
  par_for(0, M.nr, [&](int64_t i) {
    double q = 0.0, a = 0.0;
    if (Qm && Qm->nnz() > 0)
      for (int64_t k = Qm->rp[i]; k < Qm->rp[i + 1]; ++k)
        q = use_sum ? q + std::fabs(Qm->v[k]) : std::max(q, std::fabs(Qm->v[k]));
    for (int64_t k = M.rp[i]; k < M.rp[i + 1]; ++k)
      a = use_sum ? a + std::fabs(M.v[k]) : std::max(a, std::fabs(M.v[k]));
    double r = use_sum ? q + a : std::max(q, a);
    outv[i] = clip4(r > 0.0 ? std::sqrt(r) : 1.0);
  }, 1024);
}

// scale_csr_row_col_kernel! (kernels.jl:7120-7140): v * (1/r_i) / c_j
void scale_csr(CSR& M, const vector<double>& r, const vector<double>& cl) {
  par_for(0, M.nr, [&](int64_t i) {
    double rinv = 1.0 / r[i];
    for (int64_t k = M.rp[i]; k < M.rp[i + 1]; ++k) {
      double v = M.v[k];
      v *= rinv;
      v /= cl[M.ci[k]];
      M.v[k] = v;
    }
  }, 1024);
}

double bound_norm_pair_l2(const vector<double>& AL, const vector<double>& AU,
                          bool inf_norm) {
  // max.(abs.(AL_nInf), abs.(AU_nInf)) with infinite entries zeroed
  int64_t m = (int64_t)AL.size();
  if (inf_norm) {
    double r = 0;
    for (int64_t i = 0; i < m; ++i) {
      double a = std::isinf(AL[i]) && AL[i] < 0 ? 0.0 : AL[i];
      double b = std::isinf(AU[i]) && AU[i] > 0 ? 0.0 : AU[i];
      r = jmax(r, std::max(std::fabs(a), std::fabs(b)));
    }
    return r;
  }
  return std::sqrt(det_sum(m, [&](int64_t i) {
    double a = (AL[i] == -INF) ? 0.0 : AL[i];
    double b = (AU[i] == INF) ? 0.0 : AU[i];
    double v = std::max(std::fabs(a), std::fabs(b));
    return v * v;
  }));
}

// _finite_bound_norm (scaling.jl:621-651)
double finite_bound_norm(const vector<double>& v, int nt) {
  if (nt == HPR_BC_NORM_LINF) {
    double a = 0.0;
    for (double x : v)
      if (std::isfinite(x)) a = std::max(a, std::fabs(x));
    return a;
  }
  double a = 0.0;
  int64_t cnt = 0;
  for (double x : v)
    if (std::isfinite(x)) {
      a = std::fma(x, x, a);
      cnt++;
    }
  if (cnt == 0) return 0.0;
  if (nt == HPR_BC_NORM_RMS) return std::sqrt(a / (double)cnt);
  return std::sqrt(a);
}
// _vector_bc_norm (scaling.jl:667-676)
double vector_bc_norm(const vector<double>& v, int nt) {
  if (v.empty()) return 0.0;
  if (nt == HPR_BC_NORM_LINF) return absmax(v);
  double ss = dot(v, v);
  if (nt == HPR_BC_NORM_RMS) return std::sqrt(ss / (double)v.size());
  return std::sqrt(ss);
}

}  // namespace

extern "C" int oracle_scale(oracle_ctx* o, const hpr_params* prm,
                            hpr_scale_info* out) {
  int64_t m = o->m, n = o->n;
  auto soc_rhs_inf = [&]() {
    if (o->ncon() <= 0 || o->soc_rhs.empty()) return 0.0;
    return absmax(o->soc_rhs);
  };
  o->l_org = o->l;
  o->u_org = o->u;
  if (o->q_kind == HPR_Q_DIAG_LOWRANK) {
    // operator Q: no scaling at all (scaling.jl:800-846)
    o->row_norm.assign(m, 1.0);
    o->col_norm.assign(n, 1.0);
    o->norm_b_org = m > 0 ? std::max(bound_norm_pair_l2(o->AL, o->AU, true), soc_rhs_inf()) : 0.0;
    o->norm_c_org = absmax(o->c);
    o->b_scale = o->c_scale = 1.0;
    o->norm_b = m > 0 ? std::max(bound_norm_pair_l2(o->AL, o->AU, false), soc_rhs_inf()) : 0.0;
    o->norm_c = nrm2(o->c);
  } else {
    o->row_norm.assign(m, 1.0);
    o->col_norm.assign(n, 1.0);
    o->norm_b_org = std::max(bound_norm_pair_l2(o->AL, o->AU, true), soc_rhs_inf());
    o->norm_c_org = absmax(o->c);
    vector<double> tr(m, 1.0), tc(n, 1.0);
    const CSR* Qp = (o->q_kind == HPR_Q_CSR) ? &o->Q : nullptr;
    int st = prm->soc_block_scaling_strategy;
    auto apply_pass = [&](int phase, bool sum) {
      row_stat(o->AT, Qp, sum, tc);
      if (m > 0) {
        row_stat(o->A, nullptr, sum, tr);
        apply_block(tr, o->con_idx, st, phase, LOC_CON);
        for (auto& v : tr) v = clip4(v);
      }
      apply_block(tc, o->var_idx, st, phase, LOC_VAR);
      for (auto& v : tc) v = clip4(v);
      for (int64_t i = 0; i < m; ++i) o->row_norm[i] *= tr[i];
      for (int64_t i = 0; i < n; ++i) o->col_norm[i] *= tc[i];
      if (Qp) scale_csr(o->Q, tc, tc);
      if (m > 0) {
        scale_csr(o->A, tr, tc);
        scale_csr(o->AT, tc, tr);
      }
      for (int64_t i = 0; i < n; ++i) o->c[i] /= tc[i];
      if (m > 0) {
        for (int64_t i = 0; i < m; ++i) {
          o->AL[i] /= tr[i];
          o->AU[i] /= tr[i];
        }
        if (!o->soc_rhs.empty()) {
          for (int64_t i = o->m_lin; i < m; ++i) o->soc_rhs[i - o->m_lin] /= tr[i];
          for (int64_t i = 0; i < m; ++i) o->soc_rhs_full[i] /= tr[i];
        }
      }
      for (int64_t i = 0; i < n; ++i) {
        o->l[i] *= tc[i];
        o->u[i] *= tc[i];
      }
    };
    if (prm->use_Ruiz_scaling)
      for (int it = 0; it < std::max(prm->ruiz_iterations, 0); ++it) apply_pass(PH_RUIZ, false);
    if (uses_pre_pock(st))
      for (int it = 0; it < 2; ++it) apply_pass(PH_PRE_POCK, false);
    if (prm->use_Pock_Chambolle_scaling) apply_pass(PH_POCK, true);
    if (prm->use_bc_scaling) {
      // compute_bc_scales (scaling.jl:722-729)
      int nt = prm->bc_scaling_norm_type;
      double srhs = (o->ncon() <= 0 || o->soc_rhs.empty()) ? 0.0 : vector_bc_norm(o->soc_rhs, nt);
      double hb = clip4(std::max({1.0, finite_bound_norm(o->AL, nt), finite_bound_norm(o->AU, nt), srhs}));
      double hc = clip4(std::max(1.0, vector_bc_norm(o->c, nt)));
      double sb = hb;
      double sc = jclamp(hc, hb / 1e2, hb / 1e-2);
      if (Qp) {
        double f = sb / sc;
        for (auto& v : o->Q.v) v *= f;
      }
      if (m > 0) {
        for (int64_t i = 0; i < m; ++i) {
          o->AL[i] /= sb;
          o->AU[i] /= sb;
        }
        if (!o->soc_rhs.empty()) {
          for (auto& v : o->soc_rhs) v /= sb;
          for (auto& v : o->soc_rhs_full) v /= sb;
        }
      }
      for (auto& v : o->c) v /= sc;
      for (int64_t i = 0; i < n; ++i) {
        o->l[i] /= sb;
        o->u[i] /= sb;
      }
      o->b_scale = sb;
      o->c_scale = sc;
    } else {
      o->b_scale = o->c_scale = 1.0;
    }
    o->norm_b = std::max(bound_norm_pair_l2(o->AL, o->AU, false), soc_rhs_inf());
    o->norm_c = nrm2(o->c);
  }
  // _finalize_soc_scalar_scales! (scaling.jl:551-566)
  for (int64_t i = 0; i < o->ncon(); ++i) {
    double mx = 0;
    for (int64_t j = o->con_idx[i]; j < o->con_idx[i + 1]; ++j) mx = std::max(mx, o->row_norm[j]);
    o->soc_con_scale[i] = 1.0 / (mx * o->b_scale);
  }
  for (int64_t i = 0; i < o->nvar(); ++i) {
    double mx = 0;
    for (int64_t j = o->var_idx[i]; j < o->var_idx[i + 1]; ++j) mx = std::max(mx, o->col_norm[j]);
    o->soc_var_scale[i] = 1.0 / (mx * o->c_scale);
  }
  // check_Q_diagonal (scaling.jl:1327-1353, GPU form)
  o->diag_Q.assign(n, 0.0);
  if (o->q_kind == HPR_Q_CSR || o->q_kind == HPR_Q_NONE) {
    bool isd = true;
    double dev = 0.0;
    if (o->q_kind == HPR_Q_CSR) {
      for (int64_t i = 0; i < n; ++i) {
        int64_t a = o->Q.rp[i], b = o->Q.rp[i + 1];
        if (b - a == 1) isd = isd && (o->Q.ci[a] == i);
        else if (b - a > 1) isd = false;
        double rs = 0.0;
        for (int64_t k = a; k < b; ++k) {
          rs += std::fabs(o->Q.v[k]);
          if (o->Q.ci[k] == i) o->diag_Q[i] = o->Q.v[k];
        }
        dev = std::max(dev, std::fabs(rs - std::fabs(o->diag_Q[i])));
      }
    }
    o->Q_is_diag = isd && dev <= 1e-10;
  } else {
    o->Q_is_diag = false;
  }
  o->scaled = true;
  if (out) {
    out->b_scale = o->b_scale;
    out->c_scale = o->c_scale;
    out->norm_b = o->norm_b;
    out->norm_c = o->norm_c;
    out->norm_b_org = o->norm_b_org;
    out->norm_c_org = o->norm_c_org;
    out->Q_is_diag = o->Q_is_diag ? 1 : 0;
  }
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// Power iteration (eigenvalues.jl:68-196)
// ---------------------------------------------------------------------------
extern "C" int oracle_power_A(oracle_ctx* o, int maxit, double tol,
                              double* lam) {
  int64_t m = o->m, n = o->n;
  if (m == 0) {
    *lam = 0.0;
    return HPR_OK;
  }
  vector<double> z(m), q(m), ATq(n);
  start_vector(z, 1);
  double lambda = 1.0;
  for (int it = 0; it < maxit; ++it) {
    double nz = nrm2(z);
    for (int64_t i = 0; i < m; ++i) q[i] = z[i] / nz;
    spmv(o->AT, q.data(), ATq.data());
    spmv(o->A, ATq.data(), z.data());
    lambda = dot(q, z);
    for (int64_t i = 0; i < m; ++i) q[i] = z[i] - lambda * q[i];
    double err = nrm2(q) / (nrm2(z) + lambda);
    if (err < tol) break;
  }
  *lam = lambda;
  return HPR_OK;
}

extern "C" int oracle_power_Q(oracle_ctx* o, int maxit, double tol,
                              double* lam) {
  int64_t n = o->n;
  if (!o->has_q || n == 0) {
    *lam = 0.0;
    return HPR_OK;
  }
  vector<double> z(n), q(n);
  start_vector(z, 1);
  double lambda = 1.0;
  for (int it = 0; it < maxit; ++it) {
    double nz = nrm2(z);
    for (int64_t i = 0; i < n; ++i) q[i] = z[i] / nz;
    o->qmap(q, z);
    lambda = dot(q, z);
    for (int64_t i = 0; i < n; ++i) q[i] = z[i] - lambda * q[i];
    double err = nrm2(q) / (nrm2(z) + lambda);
    if (err < tol) break;
  }
  *lam = lambda;
  return HPR_OK;
}

// unified_update_Q_factors! (unified_operations.jl:468-498)
static void update_q_factors(oracle_ctx* o) {
  if (!o->Q_is_diag) return;
  double s = o->sigma, s2 = s * s;
  for (int64_t i = 0; i < o->n; ++i) {
    double t2 = 1.0 / (1.0 + s * o->diag_Q[i]);
    o->fact2[i] = t2;
    o->fact[i] = s * t2;
    o->fact1[i] = s * o->diag_Q[i] * t2;
    o->fact_M[i] = s2 * t2;
  }
}

extern "C" int oracle_set_sigma_lambda(oracle_ctx* o, double sigma, double lamA,
                                       double lamQ) {
  o->sigma = sigma;
  o->lamA = lamA;
  o->lamQ = lamQ;
  update_q_factors(o);
  return HPR_OK;
}
extern "C" int oracle_set_inner(oracle_ctx* o, int64_t inner) {
  o->inner = inner;
  return HPR_OK;
}
extern "C" int oracle_get_scalars(oracle_ctx* o, double* sigma, double* lamA,
                                  double* lamQ, int64_t* inner) {
  if (sigma) *sigma = o->sigma;
  if (lamA) *lamA = o->lamA;
  if (lamQ) *lamQ = o->lamQ;
  if (inner) *inner = o->inner;
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// Iteration: no-Q path (unified_update_zx_cpu! kernels.jl:7672-7812,
// unified_update_y_noQ_cpu! kernels.jl:7817-7952) and Q path
// (update_zxw1_cpu! 7487-7664, update_y_cpu! 7976-8096, update_w2_cpu!
// 8100-8185).
// ---------------------------------------------------------------------------
namespace {

// x-side cone projection shared by both paths; z_raw is staged in z_bar like
// the reference does.  wbar_of(j, x_hat_j) gives the w_bar update (Q path).
template <class ZRAW, class WB>
void x_cones(oracle_ctx* o, double H1, double H2, ZRAW zraw, WB wbar) {
  double sigma = o->sigma;
  double* x = o->x.data();
  double* xb = o->x_bar.data();
  double* xh = o->x_hat.data();
  double* zb = o->z_bar.data();
  double* dx = o->dx.data();
  const double* lx = o->last_x.data();
  int64_t nv = o->nvar();
  par_for(0, nv, [&](int64_t k) {
    int64_t st = o->var_idx[k], en = o->var_idx[k + 1];
    double zt = zraw(st);
    zb[st] = zt;
    double ns = 0.0;
    for (int64_t j = st + 1; j < en; ++j) {
      double zj = zraw(j);
      zb[j] = zj;
      ns += zj * zj;
    }
    ns = std::sqrt(ns);
    if (ns <= -zt) {
      for (int64_t j = st; j < en; ++j) {
        xb[j] = 0.0;
        dx[j] = -x[j];
        xh[j] = -x[j];
        zb[j] = -zb[j] / sigma;
        x[j] = std::fma(H2, xh[j], H1 * lx[j]);
        wbar(j, xh[j]);
      }
    } else if (ns <= zt) {
      for (int64_t j = st; j < en; ++j) {
        double zj = zb[j];
        xb[j] = zj;
        dx[j] = zj - x[j];
        xh[j] = 2.0 * zj - x[j];
        zb[j] = 0.0;
        x[j] = std::fma(H2, xh[j], H1 * lx[j]);
        wbar(j, xh[j]);
      }
    } else {
      double pt = (ns + zt) / 2.0;
      double al = pt / ns;
      xb[st] = pt;
      dx[st] = pt - x[st];
      xh[st] = 2.0 * pt - x[st];
      zb[st] = (pt - zt) / sigma;
      x[st] = std::fma(H2, xh[st], H1 * lx[st]);
      wbar(st, xh[st]);
      for (int64_t j = st + 1; j < en; ++j) {
        double zj = zb[j];
        double pj = al * zj;
        xb[j] = pj;
        dx[j] = pj - x[j];
        xh[j] = 2.0 * pj - x[j];
        zb[j] = (pj - zj) / sigma;
        x[j] = std::fma(H2, xh[j], H1 * lx[j]);
        wbar(j, xh[j]);
      }
    }
  }, 16);
}

// y-side update on Ax (linear rows and cones), shared by both paths.
void y_update(oracle_ctx* o, double H1, double H2, bool write_ybar_partial) {
  int64_t m = o->m, ml = o->m_lin;
  double f1 = o->lamA * o->sigma;
  double f2 = 1.0 / f1;
  double* y = o->y.data();
  double* yb = o->y_bar.data();
  double* dy = o->dy.data();
  double* s = o->s.data();
  const double* Ax = o->Ax.data();
  const double* ly = o->last_y.data();
  const double* AL = o->AL.data();
  const double* AU = o->AU.data();
  bool full = o->to_check;
  par_for(0, ml, [&](int64_t i) {
    double yi = y[i];
    double sr = Ax[i] - f1 * yi;
    double sp = std::min(std::max(sr, AL[i]), AU[i]);
    double corr = sp - sr;
    double ybi = f2 * corr;
    double yh = 2.0 * ybi - yi;
    double yn = std::fma(H2, yh, H1 * ly[i]);
    if (full) {
      s[i] = sp;
      dy[i] = ybi - yi;
      yb[i] = ybi;
    } else if (write_ybar_partial) {
      yb[i] = ybi;
    }
    y[i] = yn;
  }, 1024);
  int64_t nc = o->ncon();
  const double* rhs = o->soc_rhs.data();
  int64_t c0 = nc > 0 ? o->con_idx[0] : m;
  par_for(0, nc, [&](int64_t k) {
    int64_t st = o->con_idx[k], en = o->con_idx[k + 1];
    int64_t off = st - c0;
    double t = Ax[st] - rhs[off] - f1 * y[st];
    s[st] = t;
    double ns = 0.0;
    for (int64_t j = st + 1; j < en; ++j) {
      double sj = Ax[j] - rhs[off + (j - st)] - f1 * y[j];
      s[j] = sj;
      ns += sj * sj;
    }
    ns = std::sqrt(ns);
    if (ns <= -t) {
      for (int64_t j = st; j < en; ++j) {
        double sr = s[j];
        s[j] = 0.0;
        yb[j] = f2 * (-sr);
        dy[j] = yb[j] - y[j];
        y[j] = std::fma(H2, 2.0 * yb[j] - y[j], H1 * ly[j]);
      }
    } else if (ns <= t) {
      for (int64_t j = st; j < en; ++j) {
        yb[j] = 0.0;
        dy[j] = -y[j];
        y[j] = std::fma(H2, -y[j], H1 * ly[j]);
      }
    } else {
      double pt = (ns + t) / 2.0;
      double al = pt / ns;
      s[st] = pt;
      yb[st] = f2 * (pt - t);
      dy[st] = yb[st] - y[st];
      y[st] = std::fma(H2, 2.0 * yb[st] - y[st], H1 * ly[st]);
      for (int64_t j = st + 1; j < en; ++j) {
        double sr = s[j];
        double pj = al * sr;
        s[j] = pj;
        yb[j] = f2 * (pj - sr);
        dy[j] = yb[j] - y[j];
        y[j] = std::fma(H2, 2.0 * yb[j] - y[j], H1 * ly[j]);
      }
    }
  }, 16);
}

void step_noQ(oracle_ctx* o, double H1, double H2) {
  int64_t n = o->n;
  spmv(o->AT, o->y.data(), o->ATy.data());
  double sigma = o->sigma;
  double* x = o->x.data();
  double* xb = o->x_bar.data();
  double* xh = o->x_hat.data();
  double* zb = o->z_bar.data();
  double* dx = o->dx.data();
  const double* lx = o->last_x.data();
  const double* aty = o->ATy.data();
  const double* c = o->c.data();
  const double* l = o->l.data();
  const double* u = o->u.data();
  int64_t ln = o->linear_n();
  bool full = o->to_check;
  par_for(0, ln, [&](int64_t i) {
    double xi = x[i];
    double tmp = aty[i] - c[i];
    double zr = xi + sigma * tmp;
    double xbi = std::min(std::max(zr, l[i]), u[i]);
    double xhi = 2.0 * xbi - xi;
    double xn = std::fma(H2, xhi, H1 * lx[i]);
    if (full) {
      dx[i] = xbi - xi;
      xb[i] = xbi;
      zb[i] = (xbi - zr) / sigma;
    }
    x[i] = xn;
    xh[i] = xhi;
  }, 1024);
  (void)n;
  x_cones(
      o, H1, H2, [&](int64_t j) { return x[j] + sigma * (aty[j] - c[j]); },
      [](int64_t, double) {});
  if (o->m == 0) return;
  spmv(o->A, o->x_hat.data(), o->Ax.data());
  y_update(o, H1, H2, false);
}

void step_Q(oracle_ctx* o, double H1, double H2) {
  int64_t n = o->n;
  o->qmap(o->w, o->Qw);
  bool diag = o->Q_is_diag;
  double f2s = 1.0 / (1.0 + o->sigma * o->lamQ);
  double f1s = 1.0 - f2s;
  double sigma = o->sigma;
  double* x = o->x.data();
  double* xb = o->x_bar.data();
  double* xh = o->x_hat.data();
  double* zb = o->z_bar.data();
  double* dx = o->dx.data();
  double* wb = o->w_bar.data();
  const double* w = o->w.data();
  const double* lx = o->last_x.data();
  const double* aty = o->ATy.data();
  const double* qw = o->Qw.data();
  const double* c = o->c.data();
  const double* l = o->l.data();
  const double* u = o->u.data();
  const double* F1 = o->fact1.data();
  const double* F2 = o->fact2.data();
  int64_t ln = o->linear_n();
  bool full = o->to_check;
  auto wbar = [&](int64_t i, double xhi) {
    wb[i] = diag ? std::fma(F1[i], w[i], F2[i] * xhi) : std::fma(f1s, w[i], f2s * xhi);
  };
  par_for(0, ln, [&](int64_t i) {
    double xi = x[i];
    double tmp = -qw[i] + aty[i] - c[i];
    double zr = xi + sigma * tmp;
    double xbi = std::min(std::max(zr, l[i]), u[i]);
    double xhi = 2.0 * xbi - xi;
    double xn = std::fma(H2, xhi, H1 * lx[i]);
    wbar(i, xhi);
    if (full) {
      dx[i] = xbi - xi;
      xb[i] = xbi;
      zb[i] = (xbi - zr) / sigma;
    }
    x[i] = xn;
    xh[i] = xhi;
  }, 1024);
  x_cones(
      o, H1, H2,
      [&](int64_t j) { return x[j] + sigma * (-qw[j] + aty[j] - c[j]); },
      wbar);
  // update_y_cpu!
  if (o->m > 0) {
    o->qmap(o->w_bar, o->Qw_bar);
    par_for(0, n, [&](int64_t i) {
      o->tempv[i] = o->x_hat[i] + sigma * (o->Qw[i] - o->Qw_bar[i]);
    }, 1024);
    spmv(o->A, o->tempv.data(), o->Ax.data());
    y_update(o, H1, H2, true);
  }
  // update_w2_cpu!
  spmv(o->AT, o->y_bar.data(), o->ATy_bar.data());
  double fs = sigma / (1.0 + sigma * o->lamQ);
  double* wv = o->w.data();
  double* atyv = o->ATy.data();
  const double* atyb = o->ATy_bar.data();
  const double* lw = o->last_w.data();
  const double* laty = o->last_ATy.data();
  const double* FV = o->fact.data();
  double* dw = o->dw.data();
  double* atdy = o->ATdy.data();
  par_for(0, n, [&](int64_t i) {
    double wi = wv[i];
    double wbi = wb[i];
    double ai = atyv[i];
    double abi = atyb[i];
    double f = diag ? FV[i] : fs;
    double wbn = wbi + f * (abi - ai);
    double wn = H1 * lw[i] + H2 * (2.0 * wbn - wi);
    double an = H1 * laty[i] + H2 * (2.0 * abi - ai);
    wv[i] = wn;
    atyv[i] = an;
    if (full) {
      wb[i] = wbn;
      dw[i] = wbn - wi;
      atdy[i] = abi - ai;
    }
  }, 1024);
}

}  // namespace

extern "C" int oracle_iterate(oracle_ctx* o, int64_t k, int full_last) {
  for (int64_t it = 0; it < k; ++it) {
    o->to_check = (full_last && it == k - 1);
    double H1 = 1.0 / ((double)o->inner + 2.0);
    double H2 = 1.0 - H1;
    if (o->has_q) step_Q(o, H1, H2);
    else step_noQ(o, H1, H2);
    o->inner += 1;
  }
  return HPR_OK;
}

// ---------------------------------------------------------------------------
// Residuals (compute_residuals!, algorithm.jl:113-196; compute_Rd!/Rp!,
// kernels.jl:118-292; compute_bounds_violation!, algorithm.jl:214-256)
// ---------------------------------------------------------------------------
extern "C" int oracle_residuals(oracle_ctx* o, int include_bounds,
                                hpr_residuals* r) {
  int64_t m = o->m, n = o->n;
  double bs = o->b_scale, cs = o->c_scale;
  bool skipq = !o->has_q;
  double qx_dot = 0.0;
  if (!skipq) {
    o->qmap(o->x_bar, o->Qx);
    qx_dot = dot(o->x_bar, o->Qx);
  }
  r->primal_obj_bar = bs * cs * (dot(o->c, o->x_bar) + 0.5 * qx_dot) + o->obj_constant;
  r->dual_obj_bar = bs * cs * (-0.5 * qx_dot + dot(o->z_bar, o->x_bar)) + o->obj_constant;
  if (m > 0)
    r->dual_obj_bar += bs * cs * (dot(o->y_bar, o->s) + dot(o->y_bar, o->soc_rhs_full));
  r->rel_gap_bar = std::fabs(r->primal_obj_bar - r->dual_obj_bar) /
                   (1.0 + std::max(std::fabs(r->primal_obj_bar), std::fabs(r->dual_obj_bar)));
  // dual residual in original coordinates
  if (m > 0) spmv(o->AT, o->y_bar.data(), o->ATdy.data());
  par_for(0, n, [&](int64_t i) {
    double cn = o->col_norm[i];
    double c_org = o->c[i] * cn * cs;
    double a_org = o->ATdy[i] * cn * cs;
    double z_org = o->z_bar[i] * cn * cs;
    if (skipq) {
      o->Rd[i] = c_org - a_org - z_org;
    } else {
      double q_org = o->Qx[i] * cn * cs;
      o->Rd[i] = q_org + c_org - a_org - z_org;
      o->Qx[i] = q_org;
    }
    o->ATdy[i] = a_org;
  }, 1024);
  double qx_inf = skipq ? 0.0 : absmax(o->Qx);
  r->err_Rd_org_bar = absmax(o->Rd) / (1.0 + jmax(jmax(o->norm_c_org, absmax(o->ATdy)), qx_inf));
  if (m > 0) {
    spmv(o->A, o->x_bar.data(), o->Ax.data());
    par_for(0, m, [&](int64_t i) {
      double rn = o->row_norm[i];
      double ax = o->Ax[i] * rn * bs;
      double lo = o->AL[i] * rn * bs;
      double hi = o->AU[i] * rn * bs;
      double pr = std::min(std::max(ax, lo), hi);
      o->Rp[i] = pr - ax;
      o->Ax[i] = ax;
    }, 1024);
    int64_t nc = o->ncon();
    int64_t c0 = nc > 0 ? o->con_idx[0] : m;
    par_for(0, nc, [&](int64_t k) {
      int64_t st = o->con_idx[k], en = o->con_idx[k + 1];
      int64_t off = st - c0;
      double rt = o->soc_rhs[off] * o->row_norm[st] * bs;
      double t = o->Ax[st] - rt;
      double ns = 0.0;
      for (int64_t j = st + 1; j < en; ++j) {
        double rj = o->soc_rhs[off + (j - st)] * o->row_norm[j] * bs;
        double sj = o->Ax[j] - rj;
        ns += sj * sj;
        o->Rp[j] = sj;
      }
      ns = std::sqrt(ns);
      o->Rp[st] = t;
      if (ns <= -t) {
      } else if (ns <= t) {
        for (int64_t j = st; j < en; ++j) o->Rp[j] = 0.0;
      } else {
        double f = (1 + t / ns) / 2;
        o->Rp[st] = (ns + t) / 2 - t;
        for (int64_t j = st + 1; j < en; ++j) o->Rp[j] = f * o->Rp[j] - o->Rp[j];
      }
    }, 16);
    double denom = 1.0 + jmax(o->norm_b_org, absmax(o->Ax));
    r->err_Rp_org_bar = absmax(o->Rp) / denom;
    r->err_Rp_linear_org_bar = o->m_lin > 0 ? absmax_range(o->Rp.data(), 0, o->m_lin) / denom : 0.0;
    r->err_Rp_soc_org_bar = o->m_lin < m ? absmax_range(o->Rp.data(), o->m_lin, m) / denom : 0.0;
  } else {
    r->err_Rp_org_bar = r->err_Rp_linear_org_bar = r->err_Rp_soc_org_bar = 0.0;
  }
  if (include_bounds) {
    par_for(0, n, [&](int64_t i) {
      double lv = std::max(o->l[i] - o->x_bar[i], 0.0);
      double uv = std::max(o->x_bar[i] - o->u[i], 0.0);
      o->dx[i] = (lv + uv) * (bs / o->col_norm[i]);
    }, 1024);
    int64_t nv = o->nvar();
    for (int64_t k = 0; k < nv; ++k) {
      int64_t st = o->var_idx[k], en = o->var_idx[k + 1];
      double t = o->x_bar[st];
      double ns = 0.0;
      o->dx[st] = t;
      for (int64_t j = st + 1; j < en; ++j) {
        o->dx[j] = o->x_bar[j];
        ns += o->x_bar[j] * o->x_bar[j];
      }
      ns = std::sqrt(ns);
      if (ns <= -t) {
      } else if (ns <= t) {
        for (int64_t j = st; j < en; ++j) o->dx[j] = 0.0;
      } else {
        double f = (1 + t / ns) / 2;
        o->dx[st] = (ns + t) / 2 - t;
        for (int64_t j = st + 1; j < en; ++j) o->dx[j] = f * o->dx[j] - o->dx[j];
      }
      for (int64_t j = st; j < en; ++j) o->dx[j] *= bs / o->col_norm[j];
    }
    r->err_Rp_org_bar = jmax(r->err_Rp_org_bar, absmax(o->dx));
  }
  r->KKTx_and_gap_org_bar = jmax(jmax(r->err_Rp_org_bar, r->err_Rd_org_bar), r->rel_gap_bar);
  return HPR_OK;
}

// compute_M_norm! (algorithm.jl:1302-1359)
extern "C" int oracle_mnorm(oracle_ctx* o, double* out) {
  double M1 = 0.0, M2 = (1.0 / o->sigma) * dot(o->dx, o->dx), M3 = 0.0;
  bool skipq = !o->has_q;
  double sg = o->sigma;
  if (!skipq) {
    o->qmap(o->dw, o->dQw);
    M2 -= 2.0 * dot(o->dQw, o->dx);
  }
  if (o->m > 0) {
    M1 = sg * o->lamA * dot(o->dy, o->dy);
    spmv(o->AT, o->dy.data(), o->ATdy.data());
    if (!skipq) {
      o->qmap(o->ATdy, o->QATdy);
      M1 -= 2.0 * sg * dot(o->dQw, o->ATdy);
    }
    M2 += 2.0 * dot(o->ATdy, o->dx);
    if (!skipq) {
      if (o->Q_is_diag) {
        for (int64_t i = 0; i < o->n; ++i) o->ATdy[i] *= o->fact_M[i];
        M3 = dot(o->ATdy, o->QATdy);
        M1 += sg * dot(o->dQw, o->dQw);
      } else {
        M3 = (sg * sg) / (1.0 + sg * o->lamQ) * dot(o->ATdy, o->QATdy);
        M1 += sg * o->lamQ * dot(o->dw, o->dQw);
      }
    }
  } else if (!o->Q_is_diag && !skipq) {
    M1 = sg * o->lamQ * dot(o->dw, o->dQw);
  }
  M2 += std::max(M1, 0.0);
  double M = std::max(M2, 0.0) + std::max(M3, 0.0);
  *out = std::sqrt(M);
  return HPR_OK;
}

// Inner products of update_sigma! (algorithm.jl:787-833).  Also leaves dx, dy,
// dw, dQw, ATdy, QATdy as the reference does.
extern "C" int oracle_sigma_terms(oracle_ctx* o, double* a, double* b,
                                  double* c, double* d) {
  int64_t n = o->n, m = o->m;
  bool skipq = !o->has_q;
  if (!skipq) {
    for (int64_t i = 0; i < n; ++i) o->dw[i] = o->w_bar[i] - o->last_w[i];
    o->qmap(o->dw, o->dQw);
  }
  for (int64_t i = 0; i < n; ++i) o->dx[i] = o->x_bar[i] - o->last_x[i];
  double A = 0.0, B = dot(o->dx, o->dx), C = 0.0, D = 0.0;
  if (m > 0) {
    for (int64_t i = 0; i < m; ++i) o->dy[i] = o->y_bar[i] - o->last_y[i];
    if (!skipq) {
      for (int64_t i = 0; i < n; ++i) o->ATdy[i] = o->ATy_bar[i] - o->last_ATy[i];
      o->qmap(o->ATdy, o->QATdy);
      A = o->lamA * dot(o->dy, o->dy) - 2.0 * dot(o->dQw, o->ATdy);
    } else {
      spmv(o->AT, o->dy.data(), o->ATdy.data());
      A = o->lamA * dot(o->dy, o->dy);
    }
  }
  if (!skipq) {
    if (o->Q_is_diag) {
      double nq = nrm2(o->dQw);
      A += nq * nq;
    } else {
      A += o->lamQ * dot(o->dw, o->dQw);
      if (m > 0) {
        C = dot(o->ATdy, o->QATdy);
        D = o->lamQ;
      }
    }
  }
  *a = A;
  *b = B;
  *c = C;
  *d = D;
  return HPR_OK;
}

// golden (kernels.jl:6268-6305)
extern "C" double oracle_golden(double ap, double bp, double cp, double dp,
                                double lo, double hi, double tol, int maxiter) {
  auto f = [&](double x) { return ap * x + bp / x + cp * (x * x) / (1 + dp * x); };
  double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  double a = lo, b = hi;
  double c = b - phi * (b - a);
  double d = a + phi * (b - a);
  double fc = f(c), fd = f(d);
  for (int i = 0; i < maxiter; ++i) {
    if (fd < fc) {
      a = c;
      c = d;
      fc = fd;
      d = a + phi * (b - a);
      fd = f(d);
    } else {
      b = d;
      d = c;
      fd = fc;
      c = b - phi * (b - a);
      fc = f(c);
    }
    if ((b - a) < tol) break;
  }
  return 0.5 * (a + b);
}

// unified_golden_Q_diag (unified_operations.jl:371-409): f(x) = a x + b/x +
// x^2 * dot(ATdy, QATdy ./ (1 .+ x diag_Q)).
extern "C" int oracle_sigma_golden_diag(oracle_ctx* o, double a, double b,
                                        double lo, double hi, double tol,
                                        double* out) {
  const int maxiter = 200;
  double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  auto f = [&](double x) {
    for (int64_t i = 0; i < o->n; ++i) o->tempv[i] = o->QATdy[i] / (1.0 + x * o->diag_Q[i]);
    return a * x + b / x + x * x * dot(o->ATdy, o->tempv);
  };
  double x1 = hi - phi * (hi - lo);
  double x2 = lo + phi * (hi - lo);
  double f1 = f(x1), f2 = f(x2);
  int it = 0;
  while (std::fabs(hi - lo) > tol * std::max(1.0, std::fabs(lo)) && it < maxiter) {
    if (f1 > f2) {
      lo = x1;
      x1 = x2;
      f1 = f2;
      x2 = lo + phi * (hi - lo);
      f2 = f(x2);
    } else {
      hi = x2;
      x2 = x1;
      f2 = f1;
      x1 = hi - phi * (hi - lo);
      f1 = f(x1);
    }
    it++;
  }
  *out = (f1 < f2) ? x1 : x2;
  return HPR_OK;
}

// do_restart! (algorithm.jl:1130-1166), vector part.
extern "C" int oracle_restart(oracle_ctx* o) {
  o->x = o->x_bar;
  o->last_x = o->x_bar;
  if (o->has_q) {
    o->w = o->w_bar;
    o->last_w = o->w_bar;
  }
  if (o->m > 0) {
    o->y = o->y_bar;
    o->last_y = o->y_bar;
    if (o->has_q) {
      spmv(o->AT, o->y_bar.data(), o->ATy_bar.data());
      o->last_ATy = o->ATy_bar;
      o->ATy = o->ATy_bar;
    }
  }
  o->inner = 0;
  return HPR_OK;
}

static vector<double>* vec_of(oracle_ctx* o, int which) {
  switch (which) {
    case HPR_VEC_X: return &o->x;
    case HPR_VEC_X_BAR: return &o->x_bar;
    case HPR_VEC_X_HAT: return &o->x_hat;
    case HPR_VEC_LAST_X: return &o->last_x;
    case HPR_VEC_Z_BAR: return &o->z_bar;
    case HPR_VEC_Y: return &o->y;
    case HPR_VEC_Y_BAR: return &o->y_bar;
    case HPR_VEC_LAST_Y: return &o->last_y;
    case HPR_VEC_S: return &o->s;
    case HPR_VEC_W: return &o->w;
    case HPR_VEC_W_BAR: return &o->w_bar;
    case HPR_VEC_LAST_W: return &o->last_w;
    case HPR_VEC_ATY: return &o->ATy;
    case HPR_VEC_LAST_ATY: return &o->last_ATy;
    case HPR_VEC_DX: return &o->dx;
    case HPR_VEC_DY: return &o->dy;
    case HPR_VEC_ROW_NORM: return &o->row_norm;
    case HPR_VEC_COL_NORM: return &o->col_norm;
    case HPR_VEC_C: return &o->c;
    case HPR_VEC_AL: return &o->AL;
    case HPR_VEC_AU: return &o->AU;
    case HPR_VEC_L: return &o->l;
    case HPR_VEC_U: return &o->u;
    case HPR_VEC_SOC_RHS: return &o->soc_rhs;
    case HPR_VEC_A_VALUES: return &o->A.v;
    case HPR_VEC_AT_VALUES: return &o->AT.v;
    case HPR_VEC_DW: return &o->dw;
  }
  return nullptr;
}

extern "C" int oracle_get_vector(oracle_ctx* o, int which, double* host,
                                 size_t len) {
  auto* v = vec_of(o, which);
  if (!v) return fail(o, HPR_E_BAD_INPUT, "unknown vector");
  if (v->size() != len) return fail(o, HPR_E_BAD_INPUT, "length mismatch");
  std::memcpy(host, v->data(), len * sizeof(double));
  return HPR_OK;
}

extern "C" int oracle_set_vector(oracle_ctx* o, int which, const double* host,
                                 size_t len) {
  auto* v = vec_of(o, which);
  if (!v) return fail(o, HPR_E_BAD_INPUT, "unknown vector");
  if (v->size() != len) return fail(o, HPR_E_BAD_INPUT, "length mismatch");
  std::memcpy(v->data(), host, len * sizeof(double));
  return HPR_OK;
}

// collect_results! (algorithm.jl:1222-1256)
extern "C" int oracle_get_solution(oracle_ctx* o, double* x, double* y,
                                   double* z, double* w) {
  for (int64_t i = 0; i < o->n; ++i) {
    if (x) x[i] = o->b_scale * (o->x_bar[i] / o->col_norm[i]);
    if (w) w[i] = o->has_q ? o->b_scale * (o->w_bar[i] / o->col_norm[i])
                           : o->b_scale * (o->x_bar[i] / o->col_norm[i]);
    if (z) z[i] = o->c_scale * (o->z_bar[i] * o->col_norm[i]);
  }
  if (y)
    for (int64_t i = 0; i < o->m; ++i) y[i] = o->c_scale * (o->y_bar[i] / o->row_norm[i]);
  return HPR_OK;
}

// print_step (algorithm.jl:1906-1908)
extern "C" double oracle_print_step(int64_t iter) {
  double p = std::pow(10.0, std::floor(std::log10((double)iter))) / 10.0;
  return std::max(p, 10.0);
}

// ---------------------------------------------------------------------------
// The solve loop (solve, algorithm.jl:2765-2905) with check_restart
// (1016-1099), update_sigma! (729-990) and do_restart! (1130-1166).
// ---------------------------------------------------------------------------
namespace {

struct Restart {
  int restart_flag = 0;
  bool first_restart = true;
  double last_gap = INF, current_gap = INF, save_gap = INF;
  int64_t inner = 0;
  int sufficient = 0, necessary = 0, long_ = 0, times = 0;
  double weighted_norm = INF, best_gap = INF, best_kkt = INF, best_sigma = 1.0;
  int64_t best_iter = 0;
  bool corr_active = false;
  int corr_hold = 0, corr_dir = 0;
};

bool refresh_best(double cg, double bg, double ck, double bk, int64_t bi) {
  bool improved = ck < bk;
  bool compat = cg < bg && ck <= 1.01 * bk;
  bool periodic = bi >= 10 && ck <= 1.2 * bk;
  return improved || compat || periodic;
}

void check_restart(Restart& R, int64_t iter, int64_t check_iter, double sigma,
                   double kkt) {
  R.restart_flag = 0;
  if (R.first_restart) {
    if (iter == check_iter) {
      R.first_restart = false;
      R.restart_flag = 1;
      R.weighted_norm = R.current_gap;
      R.best_gap = R.current_gap;
      R.best_kkt = kkt;
      R.best_sigma = sigma;
    }
  } else if (iter % check_iter == 0) {
    if (R.current_gap < 0) R.current_gap = 1e-6;
    if (R.current_gap <= 0.36 * R.last_gap) {
      R.sufficient++;
      R.restart_flag = 1;
    }
    if (R.current_gap <= 0.8 * R.last_gap && R.current_gap > 1.0 * R.save_gap) {
      R.necessary++;
      R.restart_flag = 2;
    }
    double fact = 0.15;
    if ((R.inner >= std::max(500.0, fact * (double)iter) ||
         (R.inner >= 10000 && R.current_gap <= 0.75 * R.last_gap)) &&
        R.current_gap > 0.9 * R.save_gap) {
      R.long_++;
      R.restart_flag = 3;
    }
    if (refresh_best(R.current_gap, R.best_gap, kkt, R.best_kkt, R.best_iter)) {
      R.best_gap = R.current_gap;
      R.best_kkt = kkt;
      R.best_sigma = sigma;
      R.best_iter = 0;
    }
    R.save_gap = R.current_gap;
  }
}

void update_sigma(oracle_ctx* o, Restart& R, const hpr_residuals& res) {
  if (R.restart_flag < 1) return;
  bool skipq = !o->has_q;
  bool has_m = o->m > 0;
  double sigma_old = o->sigma;
  const double SMIN = 1e-12, SMAX = 1e12, IMB = 1e6, FLOOR = 2.0, THR = 1e-8,
               EPS = 1e-16, LOG100 = std::log(100.0);
  double a, b, c, d;
  oracle_sigma_terms(o, &a, &b, &c, &d);
  a = std::max(a, EPS);
  b = std::max(b, EPS);
  double sm;
  if (skipq) sm = std::sqrt(b / a);
  else if (o->Q_is_diag) {
    if (has_m) oracle_sigma_golden_diag(o, a, b, 1e-12, 1e12, 1e-13, &sm);
    else sm = std::sqrt(b / a);
  } else {
    sm = has_m ? oracle_golden(a, b, c, d, 1e-12, 1e12, 1e-13, 200) : std::sqrt(b / a);
  }
  double sref = R.best_sigma;
  double ck = res.KKTx_and_gap_org_bar, cg = R.current_gap, bk = R.best_kkt, bg = R.best_gap;
  bool ref_ok = (ck <= 10.0 * bk) && (cg <= 10.0 * bg);
  double pr = std::sqrt((ck / bk) * (cg / bg));
  pr = jclamp(pr, 1.0, 10.0);
  double sbase = sm;
  if (ref_ok) {
    double theta = jclamp(std::exp(-0.3 * (pr - 1.0)), 0.0, 1.0);
    sbase = std::exp(theta * std::log(sm) + (1.0 - theta) * std::log(sref));
    sbase = jclamp(sbase, SMIN, SMAX);
  }
  double ep = std::max(res.err_Rp_org_bar, EPS);
  double ed = std::max(res.err_Rd_org_bar, EPS);
  double es = std::min(ep, ed), el = std::max(ep, ed);
  double ir = el / es;
  bool both = el <= THR;
  bool one = (es <= 0.5 * THR) && (el >= 2.0 * THR);
  bool ext = ir >= IMB;
  bool trig = !both && (one || ext);
  bool keep = !both && ((es <= 0.8 * THR) || (ir >= 0.1 * IMB));
  int dir = ed >= ep ? 1 : -1;
  if (both) {
    R.corr_active = false;
    R.corr_hold = -1;
    R.corr_dir = 0;
  } else if (trig || (R.corr_active && keep)) {
    R.corr_active = true;
    R.corr_hold = 0;
    R.corr_dir = dir;
  } else {
    R.corr_active = false;
    R.corr_hold = -1;
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
    if (R.corr_active) {
      if (R.corr_dir > 0) rk = std::max(rk, FLOOR);
      else if (R.corr_dir < 0) rk = std::min(rk, 1.0 / FLOOR);
    }
    kappa = std::exp(beta * jclamp(std::log(rk), -LOG100, LOG100));
  }
  double sn = sbase * kappa;
  if (R.corr_active) {
    if (R.corr_dir > 0) sn = std::max(sn, sigma_old * 1.5);
    else if (R.corr_dir < 0) sn = std::min(sn, sigma_old / 1.5);
  }
  sn = jclamp(sn, SMIN, SMAX);
  o->sigma = sn;
  R.best_iter += 1;
  if (o->Q_is_diag && !skipq && std::fabs(sigma_old - sn) > 1e-15) update_q_factors(o);
}

}  // namespace

extern "C" int oracle_solve(oracle_ctx* o, const hpr_params* P,
                            hpr_results* res) {
  using clk = std::chrono::steady_clock;
  auto now = [] { return std::chrono::duration<double>(clk::now().time_since_epoch()).count(); };
  if (P->sigma != -1 && !(P->sigma > 0)) return fail(o, HPR_E_BAD_INPUT, "invalid sigma");
  if (P->print_frequency != -1 && P->print_frequency <= 0)
    return fail(o, HPR_E_BAD_INPUT, "invalid print_frequency");
  hpr_scale_info si;
  if (!o->scaled) oracle_scale(o, P, &si);
  int64_t m = o->m, n = o->n;
  // sigma (allocate_workspace, algorithm.jl:1531-1551)
  double sigma;
  if (P->sigma == -1) {
    if (o->norm_c > 1e-16 && o->norm_b > 1e-16 && o->norm_b < 1e16 && o->norm_c < 1e16)
      sigma = o->norm_b / o->norm_c;
    else
      sigma = 1.0;
  } else {
    sigma = P->sigma;
  }
  double t_start = now();
  double lamA, lamQ;
  if (P->lambda_max_A > 0) lamA = P->lambda_max_A;
  else if (m > 0) {
    oracle_power_A(o, 5000, 1e-4, &lamA);
    lamA *= 1.05;
  } else lamA = 0.0;
  // compute_lambda_max_Q (unified_operations.jl:727-741)
  if (P->lambda_max_Q > 0) lamQ = P->lambda_max_Q;
  else if (!o->has_q) lamQ = 0.0;
  else if (o->q_kind == HPR_Q_DIAG_LOWRANK || !o->Q_is_diag) {
    oracle_power_Q(o, 5000, 1e-4, &lamQ);
    lamQ *= 1.05;
  } else {
    lamQ = -INF;
    for (double v : o->Q.v) lamQ = std::max(lamQ, v);
  }
  double power_time = now() - t_start;
  oracle_set_sigma_lambda(o, sigma, lamA, lamQ);
  // process_initial_points! (algorithm.jl:2612-2677)
  if (P->initial_x) {
    for (int64_t i = 0; i < n; ++i) {
      double v = P->initial_x[i] * o->col_norm[i] / o->b_scale;
      o->x[i] = o->x_bar[i] = o->last_x[i] = v;
      if (o->has_q) o->w[i] = o->w_bar[i] = o->last_w[i] = v;
    }
  }
  if (P->initial_y) {
    for (int64_t i = 0; i < m; ++i) {
      double v = P->initial_y[i];
      v = v * o->row_norm[i] / o->c_scale;
      o->y[i] = o->y_bar[i] = o->last_y[i] = v;
    }
    if (m > 0) {
      if (o->has_q) {
        spmv(o->AT, o->y_bar.data(), o->ATy_bar.data());
        o->ATy = o->ATy_bar;
        o->last_ATy = o->ATy_bar;
      } else {
        spmv(o->AT, o->y_bar.data(), o->ATy.data());
      }
    }
    if (o->has_q) o->qmap(o->x_bar, o->Qx);
    for (int64_t i = 0; i < n; ++i) {
      double tmp = o->has_q ? (-o->Qx[i] + o->ATy_bar[i] - o->c[i]) : (o->ATy[i] - o->c[i]);
      double zr = o->x_bar[i] + o->sigma * tmp;
      o->z_bar[i] = (o->x_bar[i] - zr) / o->sigma;
    }
    if (m > 0) {
      spmv(o->A, o->x_bar.data(), o->Ax.data());
      double f1 = o->lamA * o->sigma;
      for (int64_t i = 0; i < m; ++i)
        o->s[i] = std::min(std::max(o->Ax[i] - f1 * o->y[i], o->AL[i]), o->AU[i]);
    }
  }
  Restart R;
  R.best_sigma = o->sigma;
  o->inner = 0;
  hpr_residuals rs;
  std::memset(&rs, 0, sizeof(rs));
  int64_t iter_4 = 0, iter_6 = 0;
  double time_4 = 0, time_6 = 0;
  bool first_4 = true, first_6 = true;
  int64_t ci = P->check_iter;
  int status = -1;
  int64_t iter = 0;
  for (iter = 0; iter <= P->max_iter; ++iter) {
    double el = now() - t_start;
    bool print_yes;
    if (P->print_frequency == -1)
      print_yes = (std::fmod((double)iter, oracle_print_step(iter)) == 0) || iter == P->max_iter || el > P->time_limit;
    else
      print_yes = (iter % P->print_frequency == 0) || iter == P->max_iter || el > P->time_limit;
    if (iter % ci == 0 || print_yes) oracle_residuals(o, iter == 0, &rs);
    // check_break (algorithm.jl:1169-1187)
    if (rs.KKTx_and_gap_org_bar < P->stoptol) status = HPR_STATUS_OPTIMAL;
    else if (iter == P->max_iter) status = HPR_STATUS_MAX_ITER;
    else if (now() - t_start > P->time_limit) status = HPR_STATUS_TIME_LIMIT;
    check_restart(R, iter, ci, o->sigma, rs.KKTx_and_gap_org_bar);
    update_sigma(o, R, rs);
    if (R.restart_flag > 0) {
      oracle_restart(o);
      R.last_gap = R.current_gap;
      R.save_gap = INF;
      R.times++;
      R.inner = 0;
    }
    if (P->verbose && (print_yes || status >= 0))
      std::printf("%5lld    %3.2e    %3.2e    %+7.6e    %+7.6e    %3.2e    %3.2e    %6.2f\n",
                  (long long)iter, rs.err_Rp_org_bar, rs.err_Rd_org_bar, rs.primal_obj_bar,
                  rs.dual_obj_bar, rs.rel_gap_bar, o->sigma, now() - t_start);
    if (rs.KKTx_and_gap_org_bar < 1e-4 && first_4) {
      time_4 = now() - t_start;
      iter_4 = iter;
      first_4 = false;
    }
    if (rs.KKTx_and_gap_org_bar < 1e-6 && first_6) {
      time_6 = now() - t_start;
      iter_6 = iter;
      first_6 = false;
    }
    if (status >= 0) break;
    int64_t nx = iter + 1;
    bool to_check = (nx % ci == 0) || (R.restart_flag > 0);
    if (P->print_frequency == -1) to_check = to_check || (std::fmod((double)nx, oracle_print_step(nx)) == 0);
    else to_check = to_check || (nx % P->print_frequency == 0);
    // perform_iteration_step! (algorithm.jl:2722-2744)
    o->inner = R.inner;
    oracle_iterate(o, 1, to_check ? 1 : 0);
    bool need_last = R.restart_flag > 0;
    bool need_cur = (iter + 1) % ci == 0;
    if (need_last || need_cur) {
      double mn;
      oracle_mnorm(o, &mn);
      if (need_last) R.last_gap = std::min(mn, R.last_gap);
      if (need_cur) R.current_gap = mn;
    }
    R.inner += 1;
  }
  double tt = now() - t_start;
  if (res) {
    res->iter = iter;
    res->time = tt;
    res->power_time = power_time;
    res->residuals = rs.KKTx_and_gap_org_bar;
    res->primal_obj = rs.primal_obj_bar;
    res->gap = rs.rel_gap_bar;
    res->status = status;
    res->restarts = R.times;
    res->time_4 = time_4 == 0.0 ? tt : time_4;
    res->iter_4 = iter_4 == 0 ? iter : iter_4;
    res->time_6 = time_6 == 0.0 ? tt : time_6;
    res->iter_6 = iter_6 == 0 ? iter : iter_6;
    res->sigma_final = o->sigma;
    res->lambda_max_A = lamA;
    res->lambda_max_Q = lamQ;
    res->last = rs;
    oracle_get_solution(o, res->x, res->y, res->z, res->w);
  }
  return HPR_OK;
}
