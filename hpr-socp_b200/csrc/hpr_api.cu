// hpr_api.cu — the C ABI (include/hprsocp_b200.h): context, upload with
// validation, workspace, vector access and the solve loop.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <thread>

#include "hpr_engine.cuh"

#ifndef HPR_SMALL_PLAN_NNZ
#define HPR_SMALL_PLAN_NNZ 0
#endif
#ifndef HPR_MID_TILE
#define HPR_MID_TILE 704  // nonzeros per tile of a mid-size matrix (below)
#endif
#ifndef HPR_SMALL_TILE
#define HPR_SMALL_TILE 256
#endif

namespace hpr {

int set_err(Ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int dev_alloc(Ctx* c, void** p, size_t bytes) {
  // +64: tile copies round their byte ranges out to 16-byte boundaries and
  // may touch up to 15 bytes past the end of an array
  bytes = (bytes + 64 + 255) & ~(size_t)255;
  if (c->used + bytes > c->budget)
    return set_err(c, HPR_E_BUDGET,
                   "HBM budget exceeded: need " + std::to_string(c->used + bytes) + " of " + std::to_string(c->budget));
  // stream-ordered pool allocation: memory released by an earlier context of
  // this process is reused instead of being mapped again
  // (every use of the memory is ordered on c->stream, so no synchronisation
  // is needed here)
  cudaError_t e = cudaMallocAsync(p, bytes, c->stream);
  if (e != cudaSuccess) return set_err(c, HPR_E_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  c->used += bytes;
  c->allocs[*p] = bytes;
  return HPR_OK;
}

void dev_free(Ctx* c, void* p) {
  if (!p) return;
  auto it = c->allocs.find(p);
  if (it != c->allocs.end()) {
    c->used -= it->second;
    c->allocs.erase(it);
  }
  cudaFreeAsync(p, c->stream);
}

namespace {

using std::vector;

void free_all(Ctx* c) {
  auto f = [c](void* p) { dev_free(c, p); };
  for (DevCSR* M : {&c->A, &c->AT, &c->Q, &c->F, &c->FT}) {
    f(M->rowptr);
    f(M->col);
    f(M->val);
    f(M->val32);
    f(M->val16);
    *M = DevCSR();
  }
  for (Plan* p : {&c->planX, &c->planY, &c->planQ, &c->planF}) {
    f(p->d_tasks);
    f(p->d_big);
    f(p->d_lng);
    f(p->d_big_cnt);
    f(p->d_lng_cnt);
    f(p->d_partials);
    f(p->d_raw);
    f(p->d_ctr);
    f(p->d_runs);
    f(p->d_desc);
    f(p->d_cpart);
    f(p->d_bignorm);
    f(p->d_big_ready);
    f(p->d_apply_cnt);
    f(p->d_tcol);
    f(p->d_tval);
    f(p->d_tval32);
    f(p->d_tval16);
    *p = Plan();
  }
  double** vs[] = {&c->c,      &c->l,      &c->u,      &c->AL,       &c->AU,     &c->soc_rhs, &c->soc_rhs_full,
                   &c->qdiag,  &c->row_norm, &c->col_norm, &c->diag_Q, &c->fact1, &c->fact2,   &c->fact,
                   &c->fact_M, &c->x,      &c->x_hat,  &c->x_bar,    &c->last_x, &c->z_bar,   &c->dx,
                   &c->y,      &c->y_bar,  &c->last_y, &c->s,        &c->dy,     &c->w,       &c->w_bar,
                   &c->last_w, &c->dw,     &c->Qw,     &c->dQw,      &c->Qx,     &c->tempv,   &c->ATy,
                   &c->ATy_bar, &c->last_ATy, &c->ATdy, &c->QATdy,   &c->Rp,     &c->Rd,      &c->Ax,
                   &c->ftmp,   &c->ftmp2,  &c->vtmp_n, &c->vtmp_m,   &c->pz,     &c->pq,      &c->ptq,
                   &c->d_red,  &c->d_red_out, &c->d_red2};
  for (double** v : vs) {
    f(*v);
    *v = nullptr;
  }
  f(c->g32_n);
  f(c->g32_m);
  c->g32_n = c->g32_m = nullptr;
  f(c->d_con_start);
  f(c->d_var_start);
  c->d_con_start = c->d_var_start = nullptr;
  f(c->d_state);
  c->d_state = nullptr;
  f(c->qop_out);
  c->qop_out = nullptr;
  c->q_fn = nullptr;
  c->q_user = nullptr;
  c->q_lam = 0.0;
  if (c->graph_partial) cudaGraphExecDestroy(c->graph_partial);
  c->graph_partial = nullptr;
  c->graph_iters = 0;
  c->red_slots = 0;
  for (auto& kv : c->allocs) cudaFreeAsync(kv.first, c->stream);  // anything not listed above
  c->allocs.clear();
  c->used = 0;
  c->uploaded = c->scaled = false;
}

bool is_finite(double x) { return std::isfinite(x); }
bool finite_all(const double* v, int64_t n) { return host_all(v, n, is_finite); }

// A device copy of a host array (zeros for a null array) that must pass
// `check` (h2d_copy_checked); a failing value is reported with `what`
// (HPR_E_BAD_INPUT)
int put_checked(Ctx* c, double** d, const double* h, int64_t n, int check, const char* what) {
  HPR_TRY(dev_alloc_n(c, d, n));
  if (n <= 0) return HPR_OK;
  if (!h) {
    HPR_CUDA(c, cudaMemsetAsync(*d, 0, n * sizeof(double), c->stream));
    return HPR_OK;
  }
  bool ok = true;
  HPR_TRY(h2d_copy_checked(c, *d, h, (size_t)n * sizeof(double), check, &ok));
  if (!ok) return set_err(c, HPR_E_BAD_INPUT, what);
  return HPR_OK;
}

int zero_vec(Ctx* c, double** d, int64_t n) {
  HPR_TRY(dev_alloc_n(c, d, n));
  HPR_CUDA(c, cudaMemsetAsync(*d, 0, std::max<int64_t>(n, 1) * sizeof(double), c->stream));
  return HPR_OK;
}

int cone_index(Ctx* c, const int64_t* idx, int64_t len, int base, int64_t first, int64_t last, const char* name,
               vector<int64_t>& out) {
  out.clear();
  if (len <= 0 || !idx) {
    out.push_back(last);
    if (first != last) return set_err(c, HPR_E_BAD_INPUT, std::string(name) + ": empty index but rows remain");
    return HPR_OK;
  }
  for (int64_t k = 0; k < len; ++k) out.push_back(idx[k] - base);
  if (out.front() != first) return set_err(c, HPR_E_BAD_INPUT, std::string(name) + ": must start after the linear part");
  if (out.back() != last) return set_err(c, HPR_E_BAD_INPUT, std::string(name) + ": must end at the last row");
  for (int64_t k = 0; k + 1 < (int64_t)out.size(); ++k)
    if (out[k + 1] <= out[k]) return set_err(c, HPR_E_BAD_INPUT, std::string(name) + ": cone sizes must be >= 1");
  return HPR_OK;
}

const double kInf = std::numeric_limits<double>::infinity();

}  // namespace

// ---------------------------------------------------------------------------
// Host restatement of the solve loop (solve, algorithm.jl:2765-2905) with
// check_restart (1016-1099), update_sigma! (729-990) and do_restart!
// (1130-1166).  Vector work runs on the device; the host keeps the scalar
// decisions, reading back a few reductions at each check.
// ---------------------------------------------------------------------------
namespace {

struct RestartInfo {
  int flag = 0;
  bool first = true;
  double last_gap = kInf, current_gap = kInf, save_gap = kInf;
  int64_t inner = 0;
  int times = 0;
  double weighted = kInf, best_gap = kInf, best_kkt = kInf, best_sigma = 1.0;
  int64_t best_iter = 0;
  bool corr_active = false;
  int corr_dir = 0;
};

inline double jl_clamp(double x, double lo, double hi) { return x > hi ? hi : (x < lo ? lo : x); }

double print_step(int64_t iter) {
  double p = std::pow(10.0, std::floor(std::log10((double)iter))) / 10.0;
  return std::max(p, 10.0);
}

bool is_print_iter(int64_t iter, const hpr_params* P) {
  if (P->print_frequency == -1) return std::fmod((double)iter, print_step(iter)) == 0 || iter == P->max_iter;
  return iter % P->print_frequency == 0 || iter == P->max_iter;
}

void check_restart(RestartInfo& R, int64_t iter, int64_t ci, double sigma, double kkt) {
  R.flag = 0;
  if (R.first) {
    if (iter == ci) {
      R.first = false;
      R.flag = 1;
      R.weighted = R.current_gap;
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
  if ((R.inner >= std::max(500.0, 0.15 * (double)iter) || (R.inner >= 10000 && R.current_gap <= 0.75 * R.last_gap)) &&
      R.current_gap > 0.9 * R.save_gap)
    R.flag = 3;
  // should_refresh_best_sigma (algorithm.jl:690-703)
  bool improved = kkt < R.best_kkt;
  bool compat = R.current_gap < R.best_gap && kkt <= 1.01 * R.best_kkt;
  bool periodic = R.best_iter >= 10 && kkt <= 1.2 * R.best_kkt;
  if (improved || compat || periodic) {
    R.best_gap = R.current_gap;
    R.best_kkt = kkt;
    R.best_sigma = sigma;
    R.best_iter = 0;
  }
  R.save_gap = R.current_gap;
}

// golden (kernels.jl:6268-6305): golden-section search of
// a x + b/x + c x^2/(1 + d x) on [lo, hi].
double golden_search(double ap, double bp, double cp, double dp, double lo, double hi, double tol) {
  auto f = [&](double x) { return ap * x + bp / x + cp * (x * x) / (1 + dp * x); };
  const double phi = (std::sqrt(5.0) - 1.0) / 2.0;
  double a = lo, b = hi, c = b - phi * (b - a), d = a + phi * (b - a);
  double fc = f(c), fd = f(d);
  for (int i = 0; i < 200; ++i) {
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

int update_sigma(Ctx* c, RestartInfo& R, const hpr_residuals& res) {
  if (R.flag < 1) return HPR_OK;
  const bool skipq = !c->has_q, has_m = c->m > 0;
  const double s_old = c->sigma;
  double a, b, cc, d;
  HPR_TRY(launch_sigma_terms(c, &a, &b, &cc, &d));
  a = std::max(a, 1e-16);
  b = std::max(b, 1e-16);
  double sm;
  if (skipq || !has_m) sm = std::sqrt(b / a);
  else if (c->Q_is_diag) HPR_TRY(launch_golden_diag(c, a, b, 1e-12, 1e12, 1e-13, &sm));
  else sm = golden_search(a, b, cc, d, 1e-12, 1e12, 1e-13);
  // historical stabilisation (algorithm.jl:873-885)
  double ck = res.KKTx_and_gap_org_bar, cg = R.current_gap;
  bool ref_ok = (ck <= 10.0 * R.best_kkt) && (cg <= 10.0 * R.best_gap);
  double pr = jl_clamp(std::sqrt((ck / R.best_kkt) * (cg / R.best_gap)), 1.0, 10.0);
  double base = sm;
  if (ref_ok) {
    double th = jl_clamp(std::exp(-0.3 * (pr - 1.0)), 0.0, 1.0);
    base = jl_clamp(std::exp(th * std::log(sm) + (1.0 - th) * std::log(R.best_sigma)), 1e-12, 1e12);
  }
  // residual-imbalance correction (algorithm.jl:897-954)
  const double THR = 1e-8;
  double ep = std::max(res.err_Rp_org_bar, 1e-16), ed = std::max(res.err_Rd_org_bar, 1e-16);
  double es = std::min(ep, ed), el = std::max(ep, ed), ir = el / es;
  bool both = el <= THR;
  bool one = es <= 0.5 * THR && el >= 2.0 * THR;
  bool ext = ir >= 1e6;
  bool trig = !both && (one || ext);
  bool keep = !both && (es <= 0.8 * THR || ir >= 1e5);
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
    if (R.corr_active) rk = R.corr_dir > 0 ? std::max(rk, 2.0) : std::min(rk, 0.5);
    kappa = std::exp(beta * jl_clamp(std::log(rk), -std::log(100.0), std::log(100.0)));
  }
  double sn = base * kappa;
  if (R.corr_active) sn = R.corr_dir > 0 ? std::max(sn, s_old * 1.5) : std::min(sn, s_old / 1.5);
  sn = jl_clamp(sn, 1e-12, 1e12);
  c->sigma = sn;
  R.best_iter += 1;
  if (c->Q_is_diag && !skipq && std::fabs(s_old - sn) > 1e-15) HPR_TRY(update_q_factors(c));
  return push_state(c);
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Capture G partial iterations into a graph (launch-bound small problems).
int capture_partial_graph(Ctx* c, int G) {
  if (c->graph_partial) return HPR_OK;
  cudaGraph_t g;
  HPR_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HPR_OK;
  for (int i = 0; i < G && rc == HPR_OK; ++i) rc = launch_iteration(c, false);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc != HPR_OK) return rc;
  if (e != cudaSuccess) return set_err(c, HPR_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->graph_partial, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(c, HPR_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  c->graph_iters = G;
  return HPR_OK;
}

// Termination message and SOLUTION SUMMARY (handle_termination,
// algorithm.jl:1740-1790).
void print_summary(int status, const hpr_residuals& rs, int64_t iter, double solve_s, double setup_s) {
  static const char* names[] = {"OPTIMAL", "MAX_ITER", "TIME_LIMIT"};
  const char* st = (status >= 0 && status <= 2) ? names[status] : "UNKNOWN";
  if (status == HPR_STATUS_OPTIMAL) std::printf("The instance is solved, the accuracy is %.6e\n", rs.KKTx_and_gap_org_bar);
  else if (status == HPR_STATUS_MAX_ITER)
    std::printf("The maximum number of iterations is reached, the accuracy is %.6e\n", rs.KKTx_and_gap_org_bar);
  else if (status == HPR_STATUS_TIME_LIMIT)
    std::printf("The time limit is reached, the accuracy is %.6e\n", rs.KKTx_and_gap_org_bar);
  const std::string bar(80, '=');
  std::printf("\n%s\nSOLUTION SUMMARY\n%s\n", bar.c_str(), bar.c_str());
  std::printf("Status: %s\nIterations: %lld\nTime: %.2f seconds\n", st, (long long)iter, solve_s);
  std::printf("Primal Objective: %.12e\nDual Objective: %.12e\n", rs.primal_obj_bar, rs.dual_obj_bar);
  std::printf("Primal Residual: %.6e\nPrimal Residual (Linear): %.6e\nPrimal Residual (SOC): %.6e\n",
              rs.err_Rp_org_bar, rs.err_Rp_linear_org_bar, rs.err_Rp_soc_org_bar);
  std::printf("Dual Residual: %.6e\nRelative Gap: %.6e\n%s\n", rs.err_Rd_org_bar, rs.rel_gap_bar, bar.c_str());
  std::printf("Total time: %.2fs  (setup = %.2fs, solve = %.2fs)\n%s\n", setup_s + solve_s, setup_s, solve_s,
              bar.c_str());
  std::fflush(stdout);
}

// Precision of the A / A' SpMV stream (hpr_set_precision).  The reduced
// streams read FP32 / BF16 copies of the scaled values, re-packed here.
int apply_precision(Ctx* c, int mode) {
  if (mode != HPR_PREC_FP64 && mode != HPR_PREC_FP32 && mode != HPR_PREC_BF16)
    return set_err(c, HPR_E_BAD_INPUT, "unknown precision mode");
  c->precision = mode;
  if (c->graph_partial) {
    cudaGraphExecDestroy(c->graph_partial);
    c->graph_partial = nullptr;
    c->graph_iters = 0;
  }
  if (mode != HPR_PREC_FP64) HPR_TRY(repack_values(c));
  return HPR_OK;
}

}  // namespace

// Everything of `solve` before its loop: scaling, the precision of the
// stream, sigma_0, the eigenvalue estimates, the device state and the
// initial points (solve, algorithm.jl:2765-2834).
struct SolveSetup {
  double sigma = 1.0, t0 = 0.0, power_time = 0.0, scaling_s = 0.0, lamA = 0.0, lamQ = 0.0;
};

int solve_setup(Ctx* c, const hpr_params* P, SolveSetup* S) {
  if (P->sigma != -1 && !(P->sigma > 0)) return set_err(c, HPR_E_BAD_INPUT, "invalid sigma");
  if (P->print_frequency != -1 && P->print_frequency <= 0) return set_err(c, HPR_E_BAD_INPUT, "invalid print_frequency");
  if (P->check_iter <= 0) return set_err(c, HPR_E_BAD_INPUT, "invalid check_iter");
  double scaling_s = 0.0;
  if (!c->scaled) {
    const double ts = now_s();
    HPR_TRY(run_scaling(c, P, nullptr));
    scaling_s = now_s() - ts;
    if (P->verbose) std::printf("GPU SCALING time: %.2f seconds\n", scaling_s);
  }
  HPR_TRY(apply_precision(c, P->precision));
  HPR_TRY(prepare_engine(c));
  // sigma (allocate_workspace, algorithm.jl:1531-1551)
  double sigma = 1.0;
  if (P->sigma == -1) {
    if (c->norm_c > 1e-16 && c->norm_b > 1e-16 && c->norm_b < 1e16 && c->norm_c < 1e16) sigma = c->norm_b / c->norm_c;
  } else {
    sigma = P->sigma;
  }
  const double t0 = now_s();
  double lamA = 0.0, lamQ = 0.0;
  if (P->lambda_max_A > 0) lamA = P->lambda_max_A;
  else if (c->m > 0) {
    HPR_TRY(launch_power_A(c, 5000, 1e-4, &lamA));
    lamA *= 1.05;
  }
  // compute_lambda_max_Q (unified_operations.jl:727-741)
  if (P->lambda_max_Q > 0) lamQ = P->lambda_max_Q;
  else if (c->q_kind == HPR_Q_OPERATOR && c->q_lam > 0) lamQ = c->q_lam;
  else if (c->has_q) {
    if (c->q_kind == HPR_Q_DIAG_LOWRANK || !c->Q_is_diag) {
      HPR_TRY(launch_power_Q(c, 5000, 1e-4, &lamQ));
      lamQ *= 1.05;
    } else {
      vector<double> qv(c->Q.nnz);
      HPR_CUDA(c, cudaMemcpyAsync(qv.data(), c->Q.val, c->Q.nnz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      HPR_CUDA(c, cudaStreamSynchronize(c->stream));
      lamQ = -kInf;
      for (double v : qv) lamQ = std::max(lamQ, v);
    }
  }
  const double power_time = now_s() - t0;
  if (P->verbose) std::printf("ESTIMATING MAXIMUM EIGENVALUES time = %.2f seconds\n", power_time);
  c->sigma = sigma;
  c->lamA = lamA;
  c->lamQ = lamQ;
  c->inner = 0;
  HPR_TRY(push_state(c));
  HPR_TRY(update_q_factors(c));
  if (P->initial_x || P->initial_y) HPR_TRY(launch_initial_points(c, P->initial_x, P->initial_y));
  S->sigma = sigma;
  S->t0 = t0;
  S->power_time = power_time;
  S->scaling_s = scaling_s;
  S->lamA = lamA;
  S->lamQ = lamQ;
  return HPR_OK;
}

// The loop of `solve` (algorithm.jl:2835-2905) driven from the host.
int solve_host_loop(Ctx* c, const hpr_params* P, const SolveSetup& S, hpr_results* out) {
  const double t0 = S.t0, power_time = S.power_time, scaling_s = S.scaling_s, lamA = S.lamA, lamQ = S.lamQ;
  // small problems are launch-bound: replay captured partial iterations (a
  // caller's Q operator is not captured: it may not be capturable)
  if (c->A.nnz + c->n + c->m < (int64_t)4000000 && !uses_fused_iterations(c) && c->q_kind != HPR_Q_OPERATOR)
    HPR_TRY(capture_partial_graph(c, 8));
  std::unique_ptr<Checkpointer, void (*)(Checkpointer*)> ckpt(nullptr, ckpt_destroy);
  if (P->auto_save) {
    int rc = HPR_OK;
    ckpt.reset(ckpt_create(c, P, &rc));
    if (rc != HPR_OK) return rc;
  }

  RestartInfo R;
  R.best_sigma = c->sigma;
  hpr_residuals rs;
  std::memset(&rs, 0, sizeof(rs));
  int64_t iter_4 = 0, iter_6 = 0;
  double time_4 = 0, time_6 = 0;
  const int64_t ci = P->check_iter;
  int status = -1;
  int64_t iter = 0;
  // Reduced-precision stream: residuals, restart and sigma logic stay FP64;
  // the SpMV stream itself switches to FP64 for the finish once the KKT
  // measure is within `switch_factor` of the tolerance or has stopped
  // improving (no 20% gain over kStallChecks checks).  refine < 0 keeps the
  // reduced stream to the end.
  const double switch_factor = P->refine > 0 ? (double)P->refine : 10.0;
  constexpr int kStallChecks = 10;
  double red_best = kInf;
  int red_stall = 0;
  if (P->verbose) std::printf(" iter     errRp     errRd         p_obj           d_obj          gap        sigma       time\n");
  while (true) {
    // ---- the event iteration `iter` (residual check or print)
    double el = now_s() - t0;
    bool print_yes = is_print_iter(iter, P) || el > P->time_limit;
    if (iter % ci == 0 || print_yes) HPR_TRY(launch_residuals(c, iter == 0, &rs));
    if (rs.KKTx_and_gap_org_bar != rs.KKTx_and_gap_org_bar)
      return set_err(c, HPR_E_NUMERIC, "NaN in the KKT residuals at iteration " + std::to_string(iter));
    if (ckpt && (iter % ci == 0 || print_yes)) HPR_TRY(ckpt_track(ckpt.get(), iter, c->sigma, rs));
    if (rs.KKTx_and_gap_org_bar < P->stoptol) status = HPR_STATUS_OPTIMAL;
    else if (iter == P->max_iter) status = HPR_STATUS_MAX_ITER;
    else if (now_s() - t0 > P->time_limit) status = HPR_STATUS_TIME_LIMIT;
    if (c->precision != HPR_PREC_FP64 && P->refine >= 0 && status < 0 && iter > 0 && iter % ci == 0) {
      const double kkt = rs.KKTx_and_gap_org_bar;
      if (kkt < 0.8 * red_best) {
        red_best = kkt;
        red_stall = 0;
      } else {
        ++red_stall;
      }
      if (kkt < switch_factor * P->stoptol || red_stall >= kStallChecks) {
        if (P->verbose)
          std::printf("switching the SpMV stream to FP64 at iteration %lld (KKT %.2e)\n", (long long)iter, kkt);
        HPR_TRY(apply_precision(c, HPR_PREC_FP64));
        if (c->A.nnz + c->n + c->m < (int64_t)4000000 && !uses_fused_iterations(c) && c->q_kind != HPR_Q_OPERATOR)
          HPR_TRY(capture_partial_graph(c, 8));
      }
    }
    check_restart(R, iter, ci, c->sigma, rs.KKTx_and_gap_org_bar);
    HPR_TRY(update_sigma(c, R, rs));
    if (R.flag > 0) {
      HPR_TRY(launch_restart(c));
      R.last_gap = R.current_gap;
      R.save_gap = kInf;
      R.times++;
      R.inner = 0;
    }
    if (P->verbose && (print_yes || status >= 0))
      std::printf("%5lld    %3.2e    %3.2e    %+7.6e    %+7.6e    %3.2e    %3.2e    %6.2f\n", (long long)iter,
                  rs.err_Rp_org_bar, rs.err_Rd_org_bar, rs.primal_obj_bar, rs.dual_obj_bar, rs.rel_gap_bar, c->sigma,
                  now_s() - t0);
    // auto-save (algorithm.jl:2871-2880), written behind the iteration
    if (ckpt && (print_yes || status >= 0))
      HPR_TRY(ckpt_save(ckpt.get(), iter, now_s() - t0, c->sigma, rs, status >= 0));
    if (rs.KKTx_and_gap_org_bar < 1e-4 && iter_4 == 0 && time_4 == 0) {
      time_4 = now_s() - t0;
      iter_4 = iter;
      if (iter == 0) time_4 = 1e-300;
    }
    if (rs.KKTx_and_gap_org_bar < 1e-6 && iter_6 == 0 && time_6 == 0) {
      time_6 = now_s() - t0;
      iter_6 = iter;
      if (iter == 0) time_6 = 1e-300;
    }
    if (status >= 0) break;
    // ---- steps up to the next event (perform_iteration_step!, algorithm.jl:2722-2744)
    int64_t next = iter + 1;
    while (!(next % ci == 0 || is_print_iter(next, P))) ++next;
    if (R.flag > 0) {
      // the restart iteration's own step is full and needs the M-norm
      HPR_TRY(run_iterations(c, 1, true));
      double mn;
      HPR_TRY(launch_mnorm(c, &mn));
      R.last_gap = std::min(mn, R.last_gap);
      if ((iter + 1) % ci == 0) R.current_gap = mn;
      R.inner += 1;
      iter += 1;
      if (iter < next) {
        HPR_TRY(run_iterations(c, next - iter, true));
        R.inner += next - iter;
        if (next % ci == 0) HPR_TRY(launch_mnorm(c, &R.current_gap));
      }
    } else {
      HPR_TRY(run_iterations(c, next - iter, true));
      R.inner += next - iter;
      if (next % ci == 0) HPR_TRY(launch_mnorm(c, &R.current_gap));
    }
    iter = next;
  }
  const double tt = now_s() - t0;
  if (out) {
    out->iter = iter;
    out->time = tt;
    out->power_time = power_time;
    out->residuals = rs.KKTx_and_gap_org_bar;
    out->primal_obj = rs.primal_obj_bar;
    out->gap = rs.rel_gap_bar;
    out->status = status;
    out->restarts = R.times;
    out->time_4 = time_4 == 0.0 ? tt : (time_4 < 1e-200 ? 0.0 : time_4);
    out->iter_4 = (iter_4 == 0 && time_4 == 0.0) ? iter : iter_4;
    out->time_6 = time_6 == 0.0 ? tt : (time_6 < 1e-200 ? 0.0 : time_6);
    out->iter_6 = (iter_6 == 0 && time_6 == 0.0) ? iter : iter_6;
    out->sigma_final = c->sigma;
    out->lambda_max_A = lamA;
    out->lambda_max_Q = lamQ;
    out->last = rs;
    HPR_TRY(launch_unscale(c, out->x, out->y, out->z, out->w));
  }
  if (ckpt) ckpt_finish(ckpt.get());
  if (P->verbose) print_summary(status, rs, iter, tt, c->upload_s + scaling_s);
  return HPR_OK;
}

int solve_loop(Ctx* c, const hpr_params* P, hpr_results* out) {
  SolveSetup S;
  HPR_TRY(solve_setup(c, P, &S));
  return solve_host_loop(c, P, S, out);
}

// A solve whose loop runs on the device (one CTA of the request loop) when
// the problem fits it, else on the host.
int solve_resident_begin(Ctx* c, const hpr_params* P, hpr_results* out, DQueue* q, ResidentJob* job,
                         bool* submitted, double* phases) {
  *submitted = false;
  SolveSetup S;
  HPR_TRY(solve_setup(c, P, &S));
  const double t_loop = now_s();
  if (phases) {
    phases[0] = S.scaling_s;
    phases[1] = S.power_time;
  }
  if (!q || !dsolve_eligible(c, P)) {
    const int rc = solve_host_loop(c, P, S, out);
    if (phases) phases[2] = now_s() - t_loop;
    return rc;
  }
  // the device loop's clock starts after the eigenvalue estimate
  hpr_params Pd = *P;
  Pd.time_limit = P->time_limit - S.power_time;
  job->power_time = S.power_time;
  job->lamA = S.lamA;
  job->lamQ = S.lamQ;
  job->t_loop = t_loop;
  HPR_TRY(dqueue_submit(q, c, &Pd, S.sigma, &job->slot));
  *submitted = true;
  return HPR_OK;
}

int solve_resident_end(Ctx* c, const ResidentJob& job, const hpr_results& done, hpr_results* out) {
  hpr_results r = done;
  // times from the start of the eigenvalue estimate, as the host loop's
  auto shift = [&](double t) { return t + job.power_time; };
  r.time = shift(r.time);
  r.time_4 = shift(r.time_4);
  r.time_6 = shift(r.time_6);
  r.power_time = job.power_time;
  r.lambda_max_A = job.lamA;
  r.lambda_max_Q = job.lamQ;
  if (out) {
    r.x = out->x;
    r.y = out->y;
    r.z = out->z;
    r.w = out->w;
    *out = r;
    HPR_TRY(launch_unscale(c, out->x, out->y, out->z, out->w));
  }
  return HPR_OK;
}

int solve_resident(Ctx* c, const hpr_params* P, hpr_results* out, DQueue* q, double* phases) {
  ResidentJob job;
  bool submitted = false;
  HPR_TRY(solve_resident_begin(c, P, out, q, &job, &submitted, phases));
  if (!submitted) return HPR_OK;
  hpr_results r;
  std::memset(&r, 0, sizeof(r));
  int pause_us = 20;
  double t_keep = now_s();
  for (;;) {
    bool done = false;
    HPR_TRY(dqueue_poll(q, c, job.slot, &r, &done));
    if (done) break;
    std::this_thread::sleep_for(std::chrono::microseconds(pause_us));
    pause_us = std::min(2 * pause_us, 500);
    if (now_s() - t_keep > 2e-3) {
      t_keep = now_s();
      HPR_TRY(dqueue_keepalive(q) == HPR_OK ? HPR_OK : set_err(c, HPR_E_CUDA, "request loop launch failed"));
    }
  }
  return solve_resident_end(c, job, r, out);
}

}  // namespace hpr

using namespace hpr;

namespace {
Ctx* C(hpr_ctx* h) { return &h->c; }
int need_upload(Ctx* c) { return c->uploaded ? HPR_OK : set_err(c, HPR_E_STATE, "no problem uploaded"); }

int vec_ptr(Ctx* c, int which, double** p, int64_t* len) {
  const int64_t n = c->n, m = c->m;
  switch (which) {
    case HPR_VEC_X: *p = c->x; *len = n; break;
    case HPR_VEC_X_BAR: *p = c->x_bar; *len = n; break;
    case HPR_VEC_X_HAT: *p = c->x_hat; *len = n; break;
    case HPR_VEC_LAST_X: *p = c->last_x; *len = n; break;
    case HPR_VEC_Z_BAR: *p = c->z_bar; *len = n; break;
    case HPR_VEC_Y: *p = c->y; *len = m; break;
    case HPR_VEC_Y_BAR: *p = c->y_bar; *len = m; break;
    case HPR_VEC_LAST_Y: *p = c->last_y; *len = m; break;
    case HPR_VEC_S: *p = c->s; *len = m; break;
    case HPR_VEC_W: *p = c->w; *len = n; break;
    case HPR_VEC_W_BAR: *p = c->w_bar; *len = n; break;
    case HPR_VEC_LAST_W: *p = c->last_w; *len = n; break;
    case HPR_VEC_ATY: *p = c->ATy; *len = n; break;
    case HPR_VEC_LAST_ATY: *p = c->last_ATy; *len = n; break;
    case HPR_VEC_DX: *p = c->dx; *len = n; break;
    case HPR_VEC_DY: *p = c->dy; *len = m; break;
    case HPR_VEC_ROW_NORM: *p = c->row_norm; *len = m; break;
    case HPR_VEC_COL_NORM: *p = c->col_norm; *len = n; break;
    case HPR_VEC_C: *p = c->c; *len = n; break;
    case HPR_VEC_AL: *p = c->AL; *len = m; break;
    case HPR_VEC_AU: *p = c->AU; *len = m; break;
    case HPR_VEC_L: *p = c->l; *len = n; break;
    case HPR_VEC_U: *p = c->u; *len = n; break;
    case HPR_VEC_SOC_RHS: *p = c->soc_rhs; *len = m - c->m_lin; break;
    case HPR_VEC_A_VALUES: *p = c->A.val; *len = c->A.nnz; break;
    case HPR_VEC_AT_VALUES: *p = c->AT.val; *len = c->AT.nnz; break;
    case HPR_VEC_DW: *p = c->dw; *len = n; break;
    default: return set_err(c, HPR_E_BAD_INPUT, "unknown vector id");
  }
  return HPR_OK;
}
}  // namespace

namespace hpr {
namespace {
// A context's small pinned host buffers (the reduction read-back lanes and
// the state copy) are 1 KB slots of process-wide pinned slabs: a
// cudaMallocHost / cudaFreeHost pair per context costs milliseconds
// (cudaFreeHost measured 1-10 ms when a benchmark context is destroyed).
// The slabs live until the process exits.
constexpr size_t kPinSlot = 1024;
constexpr int kPinSlotsPerSlab = 256;
std::mutex g_pin_mu;
std::vector<void*> g_pin_free;

void* pin_get() {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  if (g_pin_free.empty()) {
    char* slab = nullptr;
    if (cudaHostAlloc((void**)&slab, kPinSlot * kPinSlotsPerSlab, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    for (int i = kPinSlotsPerSlab - 1; i >= 0; --i) g_pin_free.push_back(slab + (size_t)i * kPinSlot);
  }
  void* p = g_pin_free.back();
  g_pin_free.pop_back();
  return p;
}

void pin_put(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pin_free.push_back(p);
}
static_assert(64 * sizeof(double) <= kPinSlot && sizeof(DevState) <= kPinSlot, "pinned slot size");
}  // namespace
}  // namespace hpr

extern "C" {

int hpr_version(void) { return 10000; }

const char* hpr_status_string(int code) {
  switch (code) {
    case HPR_OK: return "ok";
    case HPR_E_CUDA: return "CUDA error or no usable device";
    case HPR_E_BUDGET: return "HBM budget exceeded";
    case HPR_E_BAD_INPUT: return "bad input";
    case HPR_E_NUMERIC: return "numerical failure (NaN/Inf)";
    case HPR_E_TIMEOUT: return "device wait timed out";
    case HPR_E_STATE: return "invalid call order";
    case HPR_E_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

void hpr_default_params(hpr_params* p) {
  // HPRSOCP_parameters() (src/structs.jl:277)
  std::memset(p, 0, sizeof(*p));
  p->stoptol = 1e-6;
  p->sigma = -1;
  p->max_iter = 2147483647;
  p->time_limit = 3600.0;
  p->check_iter = 150;
  p->print_frequency = -1;
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
  p->auto_save = 0;
  p->save_filename = nullptr;  // "HPRSOCP_autosave.npz"
}

int hpr_create(int device, size_t budget, hpr_ctx** out) {
  if (!out) return HPR_E_BAD_INPUT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return HPR_E_CUDA;
  if (device < 0 || device >= ndev) return HPR_E_BAD_INPUT;
  if (cudaSetDevice(device) != cudaSuccess) return HPR_E_CUDA;
  hpr_ctx* h = new hpr_ctx();
  Ctx* c = &h->c;
  c->device = device;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    delete h;
    return HPR_E_CUDA;
  }
  {
    // keep freed device memory in this process's default pool so a later
    // context reuses it; its idle part counts as free for the budget
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull, reserved = 0, inuse = 0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      // a block freed on one context's stream is not handed to another
      // context's stream behind an inserted wait on the first stream's work:
      // concurrent contexts (the serving slots) would otherwise serialise
      int no = 0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
      if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
          cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &inuse) == cudaSuccess && reserved > inuse)
        fr += (size_t)(reserved - inuse);
    }
  }
  c->budget = budget ? budget : (size_t)(0.9 * (double)fr);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      !(c->h_red_out = static_cast<double*>(pin_get())) || !(c->h_state = static_cast<DevState*>(pin_get()))) {
    pin_put(c->h_red_out);
    delete h;
    return HPR_E_CUDA;
  }
  *out = h;
  return HPR_OK;
}

int hpr_destroy(hpr_ctx* h) {
  if (!h) return HPR_OK;
  Ctx* c = C(h);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  pin_put(c->h_red_out);
  pin_put(c->h_state);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_mid) cudaEventDestroy(c->ev_mid);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete h;
  return HPR_OK;
}

const char* hpr_last_error(const hpr_ctx* h) { return h ? h->c.err.c_str() : "null context"; }

int hpr_upload(hpr_ctx* h, const hpr_problem* p) {
  if (!h || !p) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  const double t_up = now_s();
  cudaSetDevice(c->device);
  free_all(c);
  const int base = p->index_base;
  if (base != 0 && base != 1) return set_err(c, HPR_E_BAD_INPUT, "index_base must be 0 or 1");
  const int64_t m = p->m, n = p->n;
  if (m < 0 || n < 0 || p->m_lin < 0 || p->m_lin > m || p->n_box < 0 || p->n_box > n)
    return set_err(c, HPR_E_BAD_INPUT, "invalid dimensions");
  if (m > (int64_t)std::numeric_limits<int32_t>::max() - 1 || n > (int64_t)std::numeric_limits<int32_t>::max() - 1)
    return set_err(c, HPR_E_BAD_INPUT, "dimensions exceed the int32 index range");
  if ((n > 0 && (!p->c || !p->l || !p->u)) || (m > 0 && (!p->AL || !p->AU)))
    return set_err(c, HPR_E_BAD_INPUT, "null problem vector");
  c->m = m;
  c->n = n;
  c->m_lin = p->m_lin;
  c->n_box = p->n_box;
  c->obj_constant = p->obj_constant;
  if (!std::isfinite(p->obj_constant)) return set_err(c, HPR_E_BAD_INPUT, "non-finite objective constant");
  // c, the bounds, soc_rhs and q_diag are checked as they are copied to the
  // device (put_checked below)
  HPR_TRY(cone_index(c, p->soc_con_idx, p->n_soc_con_idx, base, p->m_lin, m, "soc_con_idx", c->h_con_idx));
  int64_t nbox = p->n_box;
  if (p->n_soc_var_idx > 1) {
    HPR_TRY(cone_index(c, p->soc_var_idx, p->n_soc_var_idx, base, nbox, n, "soc_var_idx", c->h_var_idx));
  } else {
    c->h_var_idx.assign(1, n);
  }
  // A and A' (validated, index-base converted and transposed on the device).
  // Each side's tile plan is host work that needs only that side's row
  // pointers, so it is built on a thread of its own while the device work,
  // the other copies and the checks go on; the threads are joined before the
  // plans are uploaded (and on every early return).
  vector<int32_t> rp, trp, qrp;
  vector<int64_t> vcones = c->h_var_idx.size() > 1 ? c->h_var_idx : vector<int64_t>();
  vector<int64_t> ccones = c->h_con_idx.size() > 1 ? c->h_con_idx : vector<int64_t>();
  int cap = 0;
  struct Joiner {
    std::vector<std::thread> t;
    ~Joiner() {
      for (auto& x : t)
        if (x.joinable()) x.join();
    }
  } plans;
  HPR_TRY(upload_csr(c, p->A, base, m, n, "A", c->A, rp));
  // problems below HPR_SMALL_PLAN_NNZ nonzeros get tiles of at most
  // HPR_SMALL_TILE nonzeros: they occupy few warps, so shorter tiles shorten
  // each launch's longest chain (0: every problem uses full tiles)
  cap = c->A.nnz < (int64_t)HPR_SMALL_PLAN_NNZ ? (int)HPR_SMALL_TILE : 0;
  // A mid-size matrix (a million nonzeros or more, but fewer than two full
  // tiles per resident warp) gets HPR_MID_TILE-nonzero tiles: its launches
  // are bound by each warp's chain of tile steps rather than by the bytes.
  // Measured on B200 on the 4.4M-nonzero Q-path instance (about 1.2 full
  // tiles per warp), iterations/s with tiles of 320 / 416 / 640 / 704 /
  // 1024 nonzeros: 6388 / 6482 / 6717 / 6781 / 6455 (means of six runs, one box).
  if (cap == 0 && c->A.nnz >= ((int64_t)1 << 20) && HPR_MID_TILE < kNnzTile) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int64_t warps = (int64_t)sms * HPR_ENGINE_MINB * kWarpsPerCta;
    if (c->A.nnz < 2 * warps * (int64_t)kNnzTile) cap = HPR_MID_TILE;
  }
  spawn_or_run(plans.t, [&] { build_plan(rp, m, ccones, c->planY, cap); });
  if (p->AT.rowptr) {
    HPR_TRY(upload_csr(c, p->AT, base, n, m, "AT", c->AT, trp));
    if (c->AT.nnz != c->A.nnz) return set_err(c, HPR_E_BAD_INPUT, "AT nnz differs from A");
  } else {
    HPR_TRY(transpose_csr(c, c->A, c->AT, trp));
  }
  spawn_or_run(plans.t, [&] { build_plan(trp, n, vcones, c->planX, cap); });
  // Q
  c->q_kind = p->q_kind;
  c->has_q = false;
  if (p->q_kind == HPR_Q_CSR) {
    HPR_TRY(upload_csr(c, p->Q, base, n, n, "Q", c->Q, qrp));
    if (c->Q.nnz == 0) {
      c->q_kind = HPR_Q_NONE;
    } else {
      c->has_q = true;
    }
  } else if (p->q_kind == HPR_Q_DIAG_LOWRANK) {
    if (!p->q_diag) return set_err(c, HPR_E_BAD_INPUT, "q_diag is null");
    int64_t k = p->F.nrows;
    vector<int32_t> frp, ftrp;
    HPR_TRY(upload_csr(c, p->F, base, k, n, "F", c->F, frp));
    HPR_TRY(transpose_csr(c, c->F, c->FT, ftrp));
    HPR_TRY(put_checked(c, &c->qdiag, p->q_diag, n, 1, "q_diag has non-finite entries"));
    c->has_q = true;
    qrp = ftrp;
    build_plan(frp, k, {}, c->planF);
    HPR_TRY(upload_plan(c, c->planF));
  } else if (p->q_kind != HPR_Q_NONE) {
    return set_err(c, HPR_E_BAD_INPUT, "unknown q_kind");
  }
  // cone index copies (int32)
  {
    vector<int32_t> cs(c->h_con_idx.begin(), c->h_con_idx.end()), vs(c->h_var_idx.begin(), c->h_var_idx.end());
    HPR_TRY(dev_alloc_n(c, &c->d_con_start, (int64_t)cs.size()));
    HPR_TRY(dev_alloc_n(c, &c->d_var_start, (int64_t)vs.size()));
    HPR_CUDA(c, cudaMemcpyAsync(c->d_con_start, cs.data(), cs.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                c->stream));
    HPR_CUDA(c, cudaMemcpyAsync(c->d_var_start, vs.data(), vs.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  if (c->has_q) spawn_or_run(plans.t, [&] { build_plan(qrp, n, vcones, c->planQ, cap); });
  // problem vectors (while the plans are being built)
  HPR_TRY(put_checked(c, &c->c, p->c, n, 1, "c has non-finite entries"));
  HPR_TRY(put_checked(c, &c->l, p->l, n, 2, "NaN in bounds"));
  HPR_TRY(put_checked(c, &c->u, p->u, n, 2, "NaN in bounds"));
  HPR_TRY(put_checked(c, &c->AL, p->AL, m, 2, "NaN in bounds"));
  HPR_TRY(put_checked(c, &c->AU, p->AU, m, 2, "NaN in bounds"));
  HPR_TRY(put_checked(c, &c->soc_rhs, p->soc_rhs, m - p->m_lin, 1, "soc_rhs has non-finite entries"));
  // plans
  for (auto& x : plans.t) x.join();
  HPR_TRY(upload_plan(c, c->planX));
  HPR_TRY(upload_plan(c, c->planY));
  if (c->has_q) HPR_TRY(upload_plan(c, c->planQ));
  // soc_rhs aligned with the rows (zero on linear rows), assembled on the device
  HPR_TRY(zero_vec(c, &c->soc_rhs_full, m));
  if (m > p->m_lin)
    HPR_CUDA(c, cudaMemcpyAsync(c->soc_rhs_full + p->m_lin, c->soc_rhs, (m - p->m_lin) * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
  // workspace (allocate_workspace, algorithm.jl:1443-1588)
  // length-n vectors (the variable side)
  double** nvecs[] = {&c->col_norm, &c->diag_Q, &c->fact1, &c->fact2, &c->fact,  &c->fact_M,
                      &c->x,        &c->x_hat,    &c->x_bar,  &c->last_x, &c->z_bar, &c->dx,   &c->w,
                      &c->w_bar,    &c->last_w,   &c->dw,     &c->Qw,     &c->dQw,   &c->Qx,   &c->tempv,
                      &c->ATy,      &c->ATy_bar,  &c->last_ATy, &c->ATdy, &c->QATdy, &c->Rd,   &c->vtmp_n,
                      &c->ptq};
  for (double** v2 : nvecs) HPR_TRY(zero_vec(c, v2, n));
  // length-m vectors (the constraint side)
  double** mvecs[] = {&c->row_norm, &c->y, &c->y_bar, &c->last_y, &c->s, &c->dy, &c->Rp, &c->Ax, &c->vtmp_m};
  for (double** v2 : mvecs) HPR_TRY(zero_vec(c, v2, m));
  HPR_TRY(zero_vec(c, &c->pz, std::max(m, n)));
  HPR_TRY(zero_vec(c, &c->pq, std::max(m, n)));
  int64_t kF = c->F.nrows;
  HPR_TRY(zero_vec(c, &c->ftmp, kF));
  HPR_TRY(zero_vec(c, &c->ftmp2, kF));
  HPR_TRY(dev_alloc_n(c, &c->g32_n, n));
  HPR_TRY(dev_alloc_n(c, &c->g32_m, m));
  HPR_TRY(zero_vec(c, &c->d_red_out, 64));
  HPR_TRY(dev_alloc_n(c, &c->d_red2, (int64_t)kWideReduceCtas * kMaxRed));
  int64_t need = (int64_t)kRedGrid * kMaxRed;
  if (need > c->red_slots) {
    dev_free(c, c->d_red);
    c->d_red = nullptr;
    HPR_TRY(dev_alloc_n(c, &c->d_red, need));
    c->red_slots = need;
  }
  {
    double *rn = c->row_norm, *cn = c->col_norm;
    HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { rn[i] = 1.0; }));
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { cn[i] = 1.0; }));
  }
  HPR_TRY(dev_alloc_n(c, &c->d_state, 1));
  c->sigma = 1.0;
  c->lamA = c->lamQ = 0.0;
  c->inner = 0;
  c->b_scale = c->c_scale = 1.0;
  c->precision = HPR_PREC_FP64;
  HPR_TRY(push_state(c));
  c->uploaded = true;
  // the arrays of the engine's tiled copies of the matrices, allocated here
  // so that nothing allocates after the upload; the first engine use after
  // the upload (normally after scaling) fills them
  HPR_TRY(prepare_engine(c, false));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  c->scaled = false;
  c->upload_s = now_s() - t_up;
  return HPR_OK;
}

int hpr_scale(hpr_ctx* h, const hpr_params* opts, hpr_scale_info* out) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (c->scaled) return set_err(c, HPR_E_STATE, "problem already scaled");
  hpr_params d;
  if (!opts) {
    hpr_default_params(&d);
    opts = &d;
  }
  cudaSetDevice(c->device);
  HPR_TRY(run_scaling(c, opts, out));
  // reduced-precision copies follow the scaled values
  if (c->precision != HPR_PREC_FP64) HPR_TRY(repack_values(c));
  return HPR_OK;
}

int hpr_power_A(hpr_ctx* h, int maxit, double tol, double* lam) {
  if (!h || !lam) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_power_A(c, maxit, tol, lam);
}

int hpr_power_Q(hpr_ctx* h, int maxit, double tol, double* lam) {
  if (!h || !lam) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_power_Q(c, maxit, tol, lam);
}

int hpr_set_sigma_lambda(hpr_ctx* h, double sigma, double lamA, double lamQ) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (!(sigma > 0) || !std::isfinite(sigma)) return set_err(c, HPR_E_BAD_INPUT, "sigma must be positive");
  c->sigma = sigma;
  c->lamA = lamA;
  c->lamQ = lamQ;
  HPR_TRY(push_state(c));
  HPR_TRY(update_q_factors(c));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

int hpr_set_inner(hpr_ctx* h, int64_t inner) {
  if (!h || inner < 0) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  c->inner = inner;
  return push_state(c);
}

int hpr_get_scalars(hpr_ctx* h, double* sigma, double* lamA, double* lamQ, int64_t* inner) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  if (sigma) *sigma = c->sigma;
  if (lamA) *lamA = c->lamA;
  if (lamQ) *lamQ = c->lamQ;
  if (inner) *inner = c->inner;
  return HPR_OK;
}

int hpr_iterate(hpr_ctx* h, int64_t k, int full_last) {
  if (!h || k < 0) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (c->m > 0 && !(c->lamA > 0)) return set_err(c, HPR_E_STATE, "lambda_A must be set before iterating");
  HPR_TRY(run_iterations(c, k, full_last != 0));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  float ms = 0;
  if (k > 0) cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  return HPR_OK;
}

int hpr_compute_residuals(hpr_ctx* h, int include_bounds, hpr_residuals* out) {
  if (!h || !out) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_residuals(c, include_bounds != 0, out);
}

int hpr_compute_residuals_noalloc(hpr_ctx* h, int include_bounds, hpr_residuals* out) {
  if (!h || !out) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, HPR_E_CUDA, "cudaSetDevice failed");
  return launch_residuals_noalloc(c, include_bounds != 0, out);
}

int hpr_mnorm(hpr_ctx* h, double* out) {
  if (!h || !out) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_mnorm(c, out);
}

int hpr_sigma_terms(hpr_ctx* h, double* a, double* b, double* cc, double* d) {
  if (!h || !a || !b || !cc || !d) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_sigma_terms(c, a, b, cc, d);
}

int hpr_sigma_golden_diag(hpr_ctx* h, double a, double b, double lo, double hi, double tol, double* out) {
  if (!h || !out) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (!c->Q_is_diag || !c->has_q) return set_err(c, HPR_E_STATE, "golden search over diag(Q) needs a diagonal Q");
  return launch_golden_diag(c, a, b, lo, hi, tol, out);
}

int hpr_restart(hpr_ctx* h) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  HPR_TRY(launch_restart(c));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

int hpr_get_vector(hpr_ctx* h, int which, double* host, size_t len) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  double* p = nullptr;
  int64_t L = 0;
  HPR_TRY(vec_ptr(c, which, &p, &L));
  if ((int64_t)len != L) return set_err(c, HPR_E_BAD_INPUT, "vector length mismatch");
  if (L > 0) {
    if (!host) return HPR_E_BAD_INPUT;
    HPR_CUDA(c, cudaMemcpyAsync(host, p, L * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  return HPR_OK;
}

int hpr_set_vector(hpr_ctx* h, int which, const double* host, size_t len) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  double* p = nullptr;
  int64_t L = 0;
  HPR_TRY(vec_ptr(c, which, &p, &L));
  if ((int64_t)len != L) return set_err(c, HPR_E_BAD_INPUT, "vector length mismatch");
  if (which == HPR_VEC_A_VALUES || which == HPR_VEC_AT_VALUES)
    if (!finite_all(host, L)) return set_err(c, HPR_E_BAD_INPUT, "non-finite matrix value");
  if (L > 0) {
    if (!host) return HPR_E_BAD_INPUT;
    HPR_CUDA(c, cudaMemcpyAsync(p, host, L * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  if (which == HPR_VEC_A_VALUES) ++c->A.version;
  if (which == HPR_VEC_AT_VALUES) ++c->AT.version;
  if (which == HPR_VEC_SOC_RHS && L > 0) {
    // the kernels read the row-aligned copy (zero on linear rows)
    HPR_CUDA(c, cudaMemcpyAsync(c->soc_rhs_full + c->m_lin, c->soc_rhs, L * sizeof(double),
                                cudaMemcpyDeviceToDevice, c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  if (c->precision != HPR_PREC_FP64 && (which == HPR_VEC_Y || which == HPR_VEC_A_VALUES || which == HPR_VEC_AT_VALUES))
    HPR_TRY(repack_values(c));
  return HPR_OK;
}

int hpr_get_solution(hpr_ctx* h, double* x, double* y, double* z, double* w) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  return launch_unscale(c, x, y, z, w);
}

int hpr_set_precision(hpr_ctx* h, int mode) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (mode != HPR_PREC_FP64 && mode != HPR_PREC_FP32 && mode != HPR_PREC_BF16)
    return set_err(c, HPR_E_BAD_INPUT, "unknown precision mode");
  return apply_precision(c, mode);
}

int hpr_device_memory(hpr_ctx* h, size_t* used_bytes, int64_t* allocations) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  if (used_bytes) *used_bytes = c->used;
  if (allocations) *allocations = (int64_t)c->allocs.size();
  return HPR_OK;
}

int hpr_set_q_operator(hpr_ctx* h, hpr_q_apply_fn apply, void* user, double lambda_max_Q) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  if (!apply) return set_err(c, HPR_E_BAD_INPUT, "null Q operator");
  if (!(lambda_max_Q >= 0.0) || !std::isfinite(lambda_max_Q))
    return set_err(c, HPR_E_BAD_INPUT, "lambda_max_Q must be finite and >= 0");
  if (c->q_kind != HPR_Q_NONE && c->q_kind != HPR_Q_OPERATOR)
    return set_err(c, HPR_E_STATE, "the uploaded problem already has a Q");
  if (c->scaled) return set_err(c, HPR_E_STATE, "set the Q operator before scaling");
  cudaSetDevice(c->device);
  const int64_t n = c->n;
  if (c->q_kind == HPR_Q_NONE) {
    // the n x n identity: the Q-path epilogues run over the operator's output
    vector<int32_t> rp((size_t)n + 1), ci((size_t)n);
    vector<double> one((size_t)n, 1.0);
    for (int64_t i = 0; i <= n; ++i) rp[i] = (int32_t)i;
    for (int64_t i = 0; i < n; ++i) ci[i] = (int32_t)i;
    hpr_csr I{n, n, n, rp.data(), ci.data(), one.data()};
    vector<int32_t> qrp;
    HPR_TRY(upload_csr(c, I, 0, n, n, "Q operator identity", c->Q, qrp));
    const vector<int64_t> vcones = c->h_var_idx.size() > 1 ? c->h_var_idx : vector<int64_t>();
    build_plan(qrp, n, vcones, c->planQ);
    HPR_TRY(upload_plan(c, c->planQ));
    HPR_TRY(dev_alloc_n(c, &c->qop_out, n));
  }
  c->q_kind = HPR_Q_OPERATOR;
  c->has_q = true;
  c->Q_is_diag = false;
  c->q_fn = apply;
  c->q_user = user;
  c->q_lam = lambda_max_Q;
  if (c->graph_partial) {
    cudaGraphExecDestroy(c->graph_partial);
    c->graph_partial = nullptr;
    c->graph_iters = 0;
  }
  HPR_TRY(prepare_engine(c));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

int hpr_set_schedule(hpr_ctx* h, int mode) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  if (mode != HPR_SCHEDULE_AUTO && mode != HPR_SCHEDULE_ENGINE && mode != HPR_SCHEDULE_FUSED)
    return set_err(c, HPR_E_BAD_INPUT, "unknown schedule");
  c->schedule = mode;
  return HPR_OK;
}

int hpr_solve(hpr_ctx* h, const hpr_params* params, hpr_results* res) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  hpr_params d;
  if (!params) {
    hpr_default_params(&d);
    params = &d;
  }
  cudaSetDevice(c->device);
  return solve_loop(c, params, res);
}

int hpr_optimize(const hpr_problem* prob, const hpr_params* params, hpr_results* res) {
  hpr_params d;
  if (!params) {
    hpr_default_params(&d);
    params = &d;
  }
  hpr_ctx* h = nullptr;
  int rc = hpr_create(params->device_number, 0, &h);
  if (rc != HPR_OK) return rc;
  rc = hpr_upload(h, prob);
  if (rc == HPR_OK && params->verbose) std::printf("COPY TO GPU time: %.2f seconds\n", C(h)->upload_s);
  if (rc == HPR_OK) rc = hpr_solve(h, params, res);
  if (rc != HPR_OK && params->verbose) std::fprintf(stderr, "hpr_optimize: %s\n", hpr_last_error(h));
  hpr_destroy(h);
  return rc;
}

int hpr_last_iterate_ms(hpr_ctx* h, double* ms, int64_t* launches) {
  if (!h) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  if (ms) *ms = c->last_ms;
  if (launches) *launches = c->last_launches;
  return HPR_OK;
}

int hpr_iteration_bytes(hpr_ctx* h, double* bytes) {
  if (!h || !bytes) return HPR_E_BAD_INPUT;
  Ctx* c = C(h);
  HPR_TRY(need_upload(c));
  *bytes = iteration_bytes(c);
  return HPR_OK;
}

}  // extern "C"
