// hpr_internal.h — internal types of the B200 HPR-SOCP library.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <type_traits>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hprsocp_b200.h"

namespace hpr {

// ---------------------------------------------------------------------------
// Tiling of the fused SpMV + epilogue engine.
//   One warp processes one Task (tile) at a time: at most kNnzTile nonzeros
//   of at most kRowCap consecutive rows.  Each lane adds a contiguous run of
//   the tile's products in column order in registers (the run layout,
//   TileRun below); a row that lies inside one run is summed exactly as the
//   reference's sequential CSC/CSR accumulation, a row that spans runs adds
//   its run partials in a fixed order.
//   kThreads is the block size of the plain reduction and map kernels.
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;
// 1024 = 32 runs of 32 (the most a run's 32 row-start bits describe; with
// at most 64 rows a tile rarely holds more).  Measured on B200, the
// benchmark SOCP: 512 / 608 / 704 / 800 / 1024 nonzeros per tile give
// 3340 / 3460 / 3551 / 3583 (same box) and 704 / 1024 give 3472 / 3632
// (another box) iterations/s.
#ifndef HPR_NNZ_TILE
#define HPR_NNZ_TILE 1024
#endif
constexpr int kNnzTile = HPR_NNZ_TILE;
#ifndef HPR_ENGINE_ROWCAP
#define HPR_ENGINE_ROWCAP 64
#endif
constexpr int kRowCap = HPR_ENGINE_ROWCAP;  // 32 (one row per lane) or 64 (two)
static_assert(kRowCap == 32 || kRowCap == 64, "one or two rows per lane");
constexpr int kSmallConeMax = kRowCap;  // larger cones are split over several tiles
constexpr int kMaxRed = 8;          // reduction lanes per engine launch

enum TaskKind : int16_t {
  TASK_ROWS = 0,        // complete rows [rb,re); whole cones when cone >= 0
  TASK_CONE_PART = 1,   // complete rows inside one big cone
  TASK_LONG_PART = 2,   // a nonzero sub-range of one long row
  TASK_CONE_APPLY = 3,  // projection of rows [rb,re) of a big cone, once its norm is known
};

struct Task {
  int32_t rb, re;    // rows
  int32_t nzb, nze;  // nonzero range (empty for TASK_CONE_APPLY)
  int16_t kind;
  int16_t ncones;    // TASK_ROWS: number of whole cones in the task
  int32_t cone;      // first cone (TASK_ROWS), the cone (CONE_PART, CONE_APPLY), or -1
  int32_t group;     // big-cone slot (CONE_PART, CONE_APPLY) / long-row slot (LONG_PART)
  int32_t part;      // slice index within the long row (LONG_PART) or the big cone (CONE_PART)
};
static_assert(sizeof(Task) == 32, "Task layout");

// The run layout of a tile.  A tile of nnz nonzeros is
// cut into 32 contiguous runs of R = ceil(nnz / 32) nonzeros, run L for lane
// L, and stored lane-interleaved: element k of run L sits at slot
// sbase + 32 k + L of the plan's tiled column/value arrays, so each load of
// the warp is coalesced while every lane adds its own run in column order.
// `desc[32 t + L]` holds the row starts inside run L in its low 32 bits (bit
// k: a non-empty row begins at run element k) and, from bit kDescOrdShift,
// the number of non-empty rows that begin in runs 0..L-1.  `nonempty` marks the tile's
// non-empty rows (bit r for row rb + r).
struct TileRun {
  uint64_t nonempty;
  int32_t sbase;
  int32_t pad;
};
static_assert(sizeof(TileRun) == 16, "TileRun layout");
constexpr int kDescOrdShift = 32;
static_assert(kNnzTile <= 32 * kDescOrdShift, "a run's row-start bits must fit below kDescOrdShift");

// A cone of more than kSmallConeMax rows (or nonzeros beyond one tile) is
// split: its nparts slices (CONE_PART tiles and long rows) write the raw
// values and their share of ||tail||^2 (slot part_base + slice); the slice
// that arrives last adds the shares in slice order and publishes the norm;
// the cone's napply TASK_CONE_APPLY tiles, queued after every other tile,
// then project its rows in parallel.
struct BigCone {
  int32_t cone, rb, re, nparts;
  int32_t part_base, napply, pad0, pad1;
};
struct LongRow {
  int32_t row, nparts, partial_base, bigcone;  // bigcone slot or -1
  int32_t cpart;                               // slice index within the big cone
};

struct Plan {
  int64_t nrows = 0;
  std::vector<Task> tasks;
  std::vector<BigCone> big;
  std::vector<LongRow> lng;
  int32_t npartials = 0;  // long-row partial sums
  int32_t ncparts = 0;    // big-cone slices (norm shares)
  std::vector<TileRun> runs;   // per tile (run layout)
  std::vector<uint64_t> desc;  // per tile and lane (run layout)
  int64_t tslots = 0;          // slots of the tiled arrays (nonzeros + run padding)
  // device copies
  Task* d_tasks = nullptr;
  BigCone* d_big = nullptr;
  LongRow* d_lng = nullptr;
  int32_t* d_big_cnt = nullptr;
  int32_t* d_lng_cnt = nullptr;
  double* d_partials = nullptr;  // long-row partial sums
  double* d_raw = nullptr;       // big-cone raw values (nrows)
  int32_t* d_ctr = nullptr;      // [0] tile counter, [1] finished warps (CTAs in the static form)
  TileRun* d_runs = nullptr;
  uint64_t* d_desc = nullptr;
  double* d_cpart = nullptr;      // big-cone norm shares per slice
  double* d_bignorm = nullptr;    // published norm per big cone
  int32_t* d_big_ready = nullptr; // 1 once the norm is published (reset by the last apply tile)
  int32_t* d_apply_cnt = nullptr; // apply tiles done per big cone
  // the matrix this plan serves, in the run layout (built by ensure_tiled
  // from the CSR arrays; rebuilt when the matrix's values change)
  mutable int32_t* d_tcol = nullptr;
  mutable double* d_tval = nullptr;
  mutable float* d_tval32 = nullptr;
  mutable __nv_bfloat16* d_tval16 = nullptr;
  mutable const void* tiled_of = nullptr;  // the DevCSR the arrays were built from
  mutable int64_t tiled_version = -1;      // its value version then
  mutable int64_t tiled_version32 = -1;    // its reduced-precision version then
  int32_t nslots() const {
    return (int32_t)tasks.size() + (int32_t)big.size() + (int32_t)lng.size();
  }
};

// Build the task list of one matrix side.  `cone_starts` holds the first row
// of every cone plus an end sentinel (empty when the side has no cones);
// rows before cone_starts[0] are linear rows.
// `nnz_cap` (<= kNnzTile; 0: kNnzTile) caps the nonzeros of a tile.
void build_plan(const std::vector<int32_t>& rowptr, int64_t nrows,
                const std::vector<int64_t>& cone_starts, Plan& plan, int nnz_cap = 0);
// the run layout of the plan's tiles (called by build_plan)
void build_runs(const std::vector<int32_t>& rowptr, Plan& plan);

struct DevCSR {
  int64_t nrows = 0, ncols = 0, nnz = 0;
  int32_t* rowptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  float* val32 = nullptr;
  __nv_bfloat16* val16 = nullptr;
  int64_t version = 0;    // bumped whenever val changes (upload, scaling)
  int64_t version32 = 0;  // bumped whenever val32 / val16 are re-packed
};

// Scalars read by the kernels; lives in device memory so captured graphs stay
// valid across sigma updates and restarts.
struct DevState {
  double sigma;
  double lamA;
  double lamQ;
  double pad0;
  long long inner;
  int32_t ticket;
  int32_t error;
};

// Views of a matrix plan for a kernel launch.
struct PlanView {
  const Task* tasks;
  const BigCone* big;
  const LongRow* lng;
  int32_t* big_cnt;
  int32_t* lng_cnt;
  double* partials;
  double* raw;
  const int32_t* cone_start;  // cone start rows (+ sentinel), this side
  int32_t* task_ctr;          // next tile to take
  int32_t* done_ctr;          // warps (CTAs in the static form) that finished; the last resets both
  double* cpart;
  double* bignorm;
  int32_t* big_ready;
  int32_t* apply_cnt;
  int32_t ntasks, nbig, nlng;
  // run layout
  const TileRun* runs;
  const uint64_t* desc;
  const int32_t* tcol;
  const double* tval;
  const float* tval32;
  const __nv_bfloat16* tval16;
};

struct Ctx {
  std::string err;
  int device = 0;
  size_t budget = 0, used = 0;
  std::unordered_map<void*, size_t> allocs;  // live device allocations and their sizes
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_mid = nullptr;
  int schedule = HPR_SCHEDULE_AUTO;  // hpr_set_schedule
  bool uploaded = false, scaled = false;
  // problem
  int64_t m = 0, n = 0, m_lin = 0, n_box = 0;
  int q_kind = HPR_Q_NONE;
  bool has_q = false, Q_is_diag = false;
  DevCSR A, AT, Q, F, FT;
  std::vector<int64_t> h_con_idx, h_var_idx;  // 0-based starts + sentinel
  int32_t* d_con_start = nullptr;  // int32 copies (+ sentinel)
  int32_t* d_var_start = nullptr;
  double obj_constant = 0.0;
  Plan planX, planY, planQ, planF;
  // problem vectors (scaled in place by hpr_scale)
  double *c = nullptr, *l = nullptr, *u = nullptr, *AL = nullptr,
         *AU = nullptr, *soc_rhs = nullptr, *soc_rhs_full = nullptr,
         *qdiag = nullptr;
  // scaling
  double *row_norm = nullptr, *col_norm = nullptr;
  double b_scale = 1, c_scale = 1, norm_b = 0, norm_c = 0, norm_b_org = 0,
         norm_c_org = 0;
  double* diag_Q = nullptr;
  double *fact1 = nullptr, *fact2 = nullptr, *fact = nullptr,
         *fact_M = nullptr;
  // workspace
  double *x = nullptr, *x_hat = nullptr, *x_bar = nullptr, *last_x = nullptr,
         *z_bar = nullptr, *dx = nullptr;
  double *y = nullptr, *y_bar = nullptr, *last_y = nullptr, *s = nullptr,
         *dy = nullptr;
  double *w = nullptr, *w_bar = nullptr, *last_w = nullptr, *dw = nullptr,
         *Qw = nullptr, *dQw = nullptr, *Qx = nullptr, *tempv = nullptr;
  double *ATy = nullptr, *ATy_bar = nullptr, *last_ATy = nullptr,
         *ATdy = nullptr, *QATdy = nullptr;
  double *Rp = nullptr, *Rd = nullptr, *Ax = nullptr;
  double* ftmp = nullptr;   // F v (k)
  double* ftmp2 = nullptr;  // F w_bar (k)
  double* vtmp_n = nullptr;
  // user Q operator (HPR_Q_OPERATOR): Q v by the caller's callback into
  // qop_out; Q / planQ hold the n x n identity so that the Q-path epilogues
  // run over the callback's output
  hpr_q_apply_fn q_fn = nullptr;
  void* q_user = nullptr;
  double q_lam = 0.0;
  double* qop_out = nullptr;
  // the device-resident loop's split of its last solve: seconds in
  // iterations, residual checks, M-norms, sigma updates, restarts; checks
  double dloop[6] = {0, 0, 0, 0, 0, 0};
  double* vtmp_m = nullptr;
  float* g32_n = nullptr;  // FP32 copies of gathered vectors (x_hat/tempv, y)
  float* g32_m = nullptr;
  double *pz = nullptr, *pq = nullptr, *ptq = nullptr;  // power iteration
  // reductions
  double* d_red = nullptr;      // partial slots
  int64_t red_slots = 0;
  double* d_red_out = nullptr;  // final results (kMaxRed * 2)
  double* d_red2 = nullptr;     // chunk sums of a two-level slot reduction (148 slots)
  double* h_red_out = nullptr;  // pinned
  DevState* d_state = nullptr;
  DevState* h_state = nullptr;  // pinned staging
  // host mirrors
  double sigma = 1, lamA = 0, lamQ = 0;
  int64_t inner = 0;
  int precision = HPR_PREC_FP64;
  // graphs
  cudaGraphExec_t graph_partial = nullptr;
  int graph_iters = 0;
  // timing
  double last_ms = 0;
  double upload_s = 0;  // wall time of the last hpr_upload (COPY TO GPU time)
  int64_t last_launches = 0;
  int64_t launches = 0;
};

// error helpers
int set_err(Ctx* c, int code, const std::string& msg);
// (a failed call's error is also taken off the runtime's last-error slot, so
// a later cudaGetLastError() check does not report it again)
#define HPR_CUDA(ctx, call)                                                 \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      (void)cudaGetLastError();                                             \
      return ::hpr::set_err((ctx), HPR_E_CUDA,                              \
                            std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                       \
  } while (0)
#define HPR_TRY(...)                 \
  do {                               \
    int rc_ = (__VA_ARGS__);         \
    if (rc_ != HPR_OK) return rc_;   \
  } while (0)

int dev_alloc(Ctx* c, void** p, size_t bytes);
void dev_free(Ctx* c, void* p);  // stream-ordered; tolerates null
template <class T>
int dev_alloc_n(Ctx* c, T** p, int64_t n) {
  return dev_alloc(c, (void**)p, (size_t)(n > 0 ? n : 1) * sizeof(T));
}

// kernel launchers (hpr_kernels.cu)
int upload_plan(Ctx* c, Plan& p);
// the plan's tiled copy of M (run layout), rebuilt when M's values changed;
// refused inside a stream capture (it may allocate)
// (build = false: only allocate the copy's arrays; its first use builds it)
int ensure_tiled(Ctx* c, const DevCSR& M, const Plan& p, bool build = true);
// ensure_tiled for every matrix side of the context
int prepare_engine(Ctx* c, bool build = true);
PlanView view_of(const Plan& p, const int32_t* cone_start);
int launch_iteration(Ctx* c, bool full);
int run_iterations(Ctx* c, int64_t k, bool full_last);
// true when run_iterations may use the single-CTA multi-iteration kernel
// (then no partial-iteration graph is captured)
bool uses_fused_iterations(const Ctx* c);
int launch_residuals(Ctx* c, bool include_bounds, hpr_residuals* out);
int launch_residuals_noalloc(Ctx* c, bool include_bounds, hpr_residuals* out);
int launch_mnorm(Ctx* c, double* out);
int launch_sigma_terms(Ctx* c, double* a, double* b, double* cc, double* d);
int launch_golden_diag(Ctx* c, double a, double b, double lo, double hi,
                       double tol, double* out);
int launch_restart(Ctx* c);
int launch_power_A(Ctx* c, int maxit, double tol, double* lam);
int launch_power_Q(Ctx* c, int maxit, double tol, double* lam);
int push_state(Ctx* c);
int update_q_factors(Ctx* c);
int launch_unscale(Ctx* c, double* x, double* y, double* z, double* w);
int launch_initial_points(Ctx* c, const double* x0, const double* y0);
int repack_values(Ctx* c);
double iteration_bytes(const Ctx* c);
// device-side CSR ingest (hpr_upload.cu): validates s, converts it to 0-based
// indices in HBM and returns the 0-based row pointers on the host
int upload_csr(Ctx* c, const hpr_csr& s, int base, int64_t nr, int64_t nc, const char* name, DevCSR& M,
               std::vector<int32_t>& rp);
// deterministic transpose on the device; trp receives T's row pointers
int transpose_csr(Ctx* c, const DevCSR& M, DevCSR& T, std::vector<int32_t>& trp);
// host-to-device copy of a pageable host array, enqueued on the context's
// stream: large arrays go through pinned chunks filled by several host
// threads (the source may be reused as soon as this returns)
int h2d_copy(Ctx* c, void* dst, const void* src, size_t bytes);
// the same for an array of doubles, checked on the way (check 1: every
// value finite, 2: no NaN); *ok is false if a value fails
int h2d_copy_checked(Ctx* c, void* dst, const void* src, size_t bytes, int check, bool* ok);
// device-to-host copy into a pageable host array after the work enqueued on
// the context's stream; returns once the data is in dst
int d2h_copy(Ctx* c, void* dst, const void* src, size_t bytes);
// pred(v[i]) for every i, checked on several host threads for long arrays
bool host_all(const double* v, int64_t n, bool (*pred)(double));
// Runs f on a new thread added to `pool`, or on the calling thread when no
// thread can be started, so that no exception leaves the library.
template <class F>
void spawn_or_run(std::vector<std::thread>& pool, F f) {
  try {
    pool.emplace_back(f);
  } catch (...) {
    f();
  }
}
// scaling (hpr_scale.cu)
int run_scaling(Ctx* c, const hpr_params* p, hpr_scale_info* out);

// device-resident solve loop and the serving request loop (hpr_dsolve.cu)
struct DQueue;
// true when the problem's whole solve loop can run in one CTA
bool dsolve_eligible(const Ctx* c, const hpr_params* P);
// the request loop on `device` with `ctas` CTAs (0: one per SM) and a ring of
// `cap` requests; null with *err set on failure
DQueue* dqueue_create(int device, int ctas, int cap, std::string* err);
void dqueue_destroy(DQueue* q);
// hand a prepared context to the request loop (non-blocking); *slot names it
int dqueue_submit(DQueue* q, Ctx* c, const hpr_params* P, double sigma0, int* slot);
// non-blocking completion check: when done, fills the scalars of `out` (not
// the vectors) and frees the slot
int dqueue_poll(DQueue* q, Ctx* c, int slot, hpr_results* out, bool* done);
// relaunch the request loop if it went idle while requests wait
int dqueue_keepalive(DQueue* q);
// submit and wait
int dqueue_solve(DQueue* q, Ctx* c, const hpr_params* P, double sigma0, hpr_results* out);

// A solve whose loop was handed to the request loop (hpr_api.cu).
struct ResidentJob {
  int slot = -1;
  double power_time = 0.0, lamA = 0.0, lamQ = 0.0, t_loop = 0.0;
};
// setup, then either hand the loop to `q` (*submitted = true, finish with
// solve_resident_end) or run the host loop to the end (*submitted = false);
// phases (may be null): wall seconds of scaling, eigenvalue estimate, loop
int solve_resident_begin(Ctx* c, const hpr_params* P, hpr_results* out, DQueue* q, ResidentJob* job,
                         bool* submitted, double* phases = nullptr);
// after dqueue_poll reported the job done: results and the unscaled solution
int solve_resident_end(Ctx* c, const ResidentJob& job, const hpr_results& r, hpr_results* out);
// solve with the loop on the device when the problem fits, waiting for it
int solve_resident(Ctx* c, const hpr_params* P, hpr_results* out, DQueue* q, double* phases = nullptr);

// auto-save of the current and best iterates (hpr_checkpoint.cu)
struct Checkpointer;
Checkpointer* ckpt_create(Ctx* c, const hpr_params* P, int* rc);
// best-iterate bookkeeping after a residual check
int ckpt_track(Checkpointer* k, int64_t iter, double sigma, const hpr_residuals& rs);
// stage the current and best iterates and hand them to the writer thread;
// a non-final save is dropped while the previous file is being written
int ckpt_save(Checkpointer* k, int64_t iter, double elapsed, double sigma, const hpr_residuals& rs, bool final);
// wait for the last file (a failed write is reported as a warning)
void ckpt_finish(Checkpointer* k);
void ckpt_destroy(Checkpointer* k);

// host-side start vector for the power iteration (splitmix64 uniform(-1,1)
// + 1e-8).  The reference uses randn(MersenneTwister(1)) .+ 1e-8
// (src/utils/eigenvalues.jl:72-76), which has no portable equivalent.
void power_start_vector(std::vector<double>& z, uint64_t seed);

}  // namespace hpr

struct hpr_ctx {
  hpr::Ctx c;
};
