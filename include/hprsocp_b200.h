/*
 * hprsocp_b200.h — C ABI of the B200 (sm_100a) dual Halpern Peaceman–Rachford
 * (HPR) iteration for convex quadratic second-order cone programs
 *
 *     min  1/2 x'Qx + c'x
 *     s.t. AL <= A1 x <= AU,   A2 x - b2 in K_soc,   l <= x1 <= u,   x2 in K_var.
 *
 * The problem is given in the reference solver's canonical ordering
 * (src/utils/builders.jl:8-22 of PolyU-IOR/HPR-SOCP): linear rows of A first
 * (equalities, then inequalities), second-order-cone rows last; boxed variables
 * first, cone variables last, each cone contiguous.  Cone blocks are described
 * by start-index vectors exactly like the reference's `SOC_con_idx` /
 * `SOC_var_idx` (src/structs.jl:139-149), in either 0- or 1-based form.
 *
 * Everything crossing this boundary is plain C: pointers, sizes and status
 * codes.  No C++ exception, CUDA type or torch type appears here.  The library
 * copies every host array it is given; it owns all device memory until
 * hpr_destroy().  There is no CPU fallback: without a usable CUDA device every
 * call returns HPR_E_CUDA.
 *
 * Each entry point names the reference function whose device-side role it
 * takes over (file:line within the reference project).
 */
#ifndef HPRSOCP_B200_H
#define HPRSOCP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define HPR_OK 0
#define HPR_E_CUDA 1      /* CUDA runtime error or no usable device          */
#define HPR_E_BUDGET 2    /* request exceeds the context's HBM budget        */
#define HPR_E_BAD_INPUT 3 /* malformed CSR, cone index, size, NaN input ...  */
#define HPR_E_NUMERIC 4   /* NaN/Inf appeared in residuals or iterates       */
#define HPR_E_TIMEOUT 5   /* a bounded device wait gave up                   */
#define HPR_E_STATE 6     /* call order violated (e.g. iterate before upload) */
#define HPR_E_UNSUPPORTED 7

/* ------------------------------------------------------------------------ */
/* Problem data                                                              */
/* ------------------------------------------------------------------------ */
typedef struct hpr_csr {
  int64_t nrows;
  int64_t ncols;
  int64_t nnz;
  const int32_t* rowptr; /* nrows+1 entries, offset by index_base          */
  const int32_t* colind; /* nnz entries, offset by index_base, sorted/row  */
  const double* values;  /* nnz entries                                    */
} hpr_csr;

/* How the quadratic term is given.
 *  NONE         : Q = 0 (the reference's "no-Q" path, has_quadratic_terms false)
 *  CSR          : explicit sparse symmetric Q; scaled with A; a diagonal CSR Q
 *                 is detected as in check_Q_diagonal (src/utils/scaling.jl:1312)
 *  DIAG_LOWRANK : operator Q = diag(q_diag) + F'F, never formed.  Like the
 *                 reference's user AbstractQOperator, an operator Q disables
 *                 all scaling (src/utils/scaling.jl:800-846).
 *  OPERATOR     : a caller-supplied Q v on the device, set after the upload
 *                 with hpr_set_q_operator (no scaling either).              */
#define HPR_Q_NONE 0
#define HPR_Q_CSR 1
#define HPR_Q_DIAG_LOWRANK 2
#define HPR_Q_OPERATOR 3

typedef struct hpr_problem {
  int64_t m;            /* rows of A                                       */
  int64_t n;            /* columns of A / variables                        */
  int64_t m_lin;        /* number_linear_con: rows 0..m_lin-1 are linear   */
  int64_t n_box;        /* number_lu_x: when variable cones exist, only    */
                        /* variables 0..n_box-1 are boxed                  */
  hpr_csr A;            /* m x n                                           */
  hpr_csr AT;           /* optional n x m transpose of A, as the reference */
                        /* keeps it (QP_info_cpu.AT); rowptr == NULL means */
                        /* "build it on upload"                            */
  const double* c;      /* n                                               */
  const double* l;      /* n (entries of cone variables are ignored)       */
  const double* u;      /* n                                               */
  const double* AL;     /* m (-inf allowed)                                */
  const double* AU;     /* m (+inf allowed)                                */
  const double* soc_rhs;/* m - m_lin: b2, aligned with the cone rows       */
  const int64_t* soc_con_idx; /* cone row starts + end sentinel           */
  int64_t n_soc_con_idx;      /* length (#constraint cones + 1), >= 1      */
  const int64_t* soc_var_idx; /* cone variable starts + end sentinel      */
  int64_t n_soc_var_idx;      /* length (#variable cones + 1), >= 1        */
  int32_t index_base;   /* 0 (C) or 1 (Julia) for every index above        */
  int32_t q_kind;       /* HPR_Q_*                                          */
  hpr_csr Q;            /* n x n when q_kind == HPR_Q_CSR                   */
  const double* q_diag; /* n when q_kind == HPR_Q_DIAG_LOWRANK              */
  hpr_csr F;            /* k x n factor when q_kind == HPR_Q_DIAG_LOWRANK   */
  double obj_constant;
} hpr_problem;

/* ------------------------------------------------------------------------ */
/* Parameters and results (fields mirror HPRSOCP_parameters and             */
/* HPRSOCP_results, src/structs.jl:208-314)                                  */
/* ------------------------------------------------------------------------ */
#define HPR_BC_NORM_L2 0
#define HPR_BC_NORM_RMS 1
#define HPR_BC_NORM_LINF 2

/* SOC block-scaling strategies (src/utils/scaling.jl:150-227).             */
#define HPR_SOC_SCALE_MAX 1
#define HPR_SOC_SCALE_RMS 2
#define HPR_SOC_SCALE_GEOM 3
#define HPR_SOC_SCALE_ADAPTIVE 4
#define HPR_SOC_SCALE_HYBRID 5
#define HPR_SOC_SCALE_RUIZ_GEOM 6
#define HPR_SOC_SCALE_ROLE_SPLIT 7
#define HPR_SOC_SCALE_POCK_SAFE_ROLE_SPLIT 8
#define HPR_SOC_SCALE_SIZE_SPLIT_ROLE_SPLIT 9
#define HPR_SOC_SCALE_PRE_POCK_SIZE_SPLIT 10
#define HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER 11
#define HPR_SOC_SCALE_PRE_POCK_HUGE_VAR_TAPER_POCK_GEOM 12
#define HPR_SOC_SCALE_PRE_POCK_BAND_SPLIT 13
#define HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_RMS 14
#define HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_MAX 15
#define HPR_SOC_SCALE_PRE_POCK_CONSTRAINT_TAPER 16
#define HPR_SOC_SCALE_SMALL_CONE_CONSTRAINT_MAX 17
#define HPR_SOC_SCALE_COUNT_AWARE_SMALL_CONE_BIAS 18
#define HPR_SOC_SCALE_PHASE_BLEND 19
#define HPR_SOC_SCALE_PHASE_TAPER 20

/* Arithmetic of the A / A' SpMV stream (hpr_set_precision).               */
#define HPR_PREC_FP64 0      /* FP64 values, FP64 accumulation (reference)  */
#define HPR_PREC_FP32 1      /* FP32 values and gathers, FP64 epilogue      */
#define HPR_PREC_BF16 2      /* BF16 values, FP32 accumulation, FP64 epilogue */

typedef struct hpr_params {
  double stoptol;        /* 1e-6                                            */
  double sigma;          /* -1 = automatic ||b||/||c|| (algorithm.jl:1538)  */
  int64_t max_iter;      /* typemax(Int32) in the reference                 */
  double time_limit;     /* seconds                                         */
  int64_t check_iter;    /* 150                                             */
  int64_t print_frequency; /* -1 = adaptive print_step (algorithm.jl:1906)  */
  int32_t device_number;
  int32_t use_Ruiz_scaling;
  int32_t ruiz_iterations;
  int32_t use_bc_scaling;
  int32_t bc_scaling_norm_type;       /* HPR_BC_NORM_*                      */
  int32_t use_Pock_Chambolle_scaling;
  int32_t soc_block_scaling_strategy; /* HPR_SOC_SCALE_*                    */
  int32_t verbose;
  const double* initial_x; /* NULL or n entries (original coordinates)    */
  const double* initial_y; /* NULL or m entries                            */
  /* Extensions (no reference counterpart): injected eigenvalue estimates
   * (values <= 0 mean "estimate by power iteration") and SpMV precision.  */
  double lambda_max_A;
  double lambda_max_Q;
  int32_t precision;       /* HPR_PREC_*                                     */
  int32_t refine;          /* reduced-precision solves: the SpMV stream
                            * switches to FP64 for the finish once the KKT
                            * measure is below refine x stoptol (refine = 0:
                            * 10 x stoptol) or stops improving; refine < 0
                            * keeps the reduced stream to the end.  Residuals,
                            * restart and sigma logic are FP64 throughout.  */
  /* Auto-save (HPRSOCP_parameters.auto_save / save_filename,
   * src/structs.jl:244-247, 271-272; written by save_state_to_hdf5!,
   * src/algorithm.jl:306-421).  When auto_save != 0, every print iteration
   * and the final iteration write the current and the best iterate (in
   * original coordinates), their residuals and these parameters to
   * save_filename (NULL or "": "HPRSOCP_autosave.npz").  The file is a NumPy
   * .npz archive whose member names are the reference's HDF5 paths
   * ("current/x_org", "best/KKTx_and_gap", "parameters/stoptol", ...); it
   * is replaced atomically and written by a background thread while the
   * iteration continues.  A failed write is a warning (verbose), not an
   * error.                                                                 */
  int32_t auto_save;
  const char* save_filename;
} hpr_params;

#define HPR_STATUS_OPTIMAL 0
#define HPR_STATUS_MAX_ITER 1
#define HPR_STATUS_TIME_LIMIT 2

typedef struct hpr_residuals {
  double err_Rp_org_bar;
  double err_Rp_linear_org_bar;
  double err_Rp_soc_org_bar;
  double err_Rd_org_bar;
  double KKTx_and_gap_org_bar;
  double primal_obj_bar;
  double rel_gap_bar;
  double dual_obj_bar;
} hpr_residuals;

typedef struct hpr_results {
  int64_t iter, iter_4, iter_6;
  double time, time_4, time_6, power_time;
  double primal_obj, residuals, gap;
  int32_t status;          /* HPR_STATUS_*                                   */
  int32_t restarts;
  double sigma_final, lambda_max_A, lambda_max_Q;
  hpr_residuals last;      /* residuals at the final check                   */
  double* x; /* caller-owned output buffers (may be NULL): n, m, n, n        */
  double* y;
  double* z;
  double* w;
} hpr_results;

typedef struct hpr_scale_info {
  double b_scale, c_scale;
  double norm_b, norm_c, norm_b_org, norm_c_org;
  int32_t Q_is_diag;
} hpr_scale_info;

/* Workspace vectors reachable through hpr_get_vector / hpr_set_vector.
 * All are in the scaled space the iteration runs in.                       */
#define HPR_VEC_X 0
#define HPR_VEC_X_BAR 1
#define HPR_VEC_X_HAT 2
#define HPR_VEC_LAST_X 3
#define HPR_VEC_Z_BAR 4
#define HPR_VEC_Y 5
#define HPR_VEC_Y_BAR 6
#define HPR_VEC_LAST_Y 7
#define HPR_VEC_S 8
#define HPR_VEC_W 9
#define HPR_VEC_W_BAR 10
#define HPR_VEC_LAST_W 11
#define HPR_VEC_ATY 12
#define HPR_VEC_LAST_ATY 13
#define HPR_VEC_DX 14
#define HPR_VEC_DY 15
#define HPR_VEC_ROW_NORM 16
#define HPR_VEC_COL_NORM 17
#define HPR_VEC_C 18          /* scaled problem data (read-only views)     */
#define HPR_VEC_AL 19
#define HPR_VEC_AU 20
#define HPR_VEC_L 21
#define HPR_VEC_U 22
#define HPR_VEC_SOC_RHS 23
#define HPR_VEC_A_VALUES 24   /* scaled A values (nnz)                     */
#define HPR_VEC_AT_VALUES 25  /* scaled A' values (nnz)                    */
#define HPR_VEC_DW 26
#define HPR_VEC_COUNT 27

typedef struct hpr_ctx hpr_ctx;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */
/* Bind a context to `device` (CUDA.device!, algorithm.jl:2771-2773) with an
 * HBM budget in bytes (0 = 90% of free memory).  Replaces the device-side
 * setup of solve() and validate_gpu_parameters! (gpu_validation.jl:16-37),
 * without its CPU fallback.                                                 */
int hpr_create(int device, size_t hbm_budget, hpr_ctx** out);
int hpr_destroy(hpr_ctx* ctx);
const char* hpr_last_error(const hpr_ctx* ctx);
const char* hpr_status_string(int code);
int hpr_version(void);

/* Copy a canonical problem to the device (transfer_to_gpu,
 * algorithm.jl:2314-2353).  Builds A' on the device, validates every index,
 * plans the fused SpMV/cone tiles (replacing the SOC bucket planner,
 * algorithm.jl:1914-2223) and allocates the workspace (allocate_workspace,
 * algorithm.jl:1443-1588).                                                  */
int hpr_upload(hpr_ctx* ctx, const hpr_problem* prob);

/* Ruiz / SOC block aggregation / Pock–Chambolle / b-c scaling on the device
 * (scaling!, src/utils/scaling.jl:785-1289) followed by check_Q_diagonal
 * (scaling.jl:1312-1353).  May be called once per upload.                   */
int hpr_scale(hpr_ctx* ctx, const hpr_params* opts, hpr_scale_info* out);

/* Power iteration for lambda_max(AA') and lambda_max(Q)
 * (power_iteration_A / _Q, src/utils/eigenvalues.jl:68-196).  Returns the
 * raw estimate; the caller applies the 1.05 safety factor like
 * estimate_eigenvalues (algorithm.jl:2434-2467).                            */
int hpr_power_A(hpr_ctx* ctx, int maxit, double tol, double* lambda_out);
int hpr_power_Q(hpr_ctx* ctx, int maxit, double tol, double* lambda_out);

/* Step size and eigenvalue bounds used by every following iteration; also
 * refreshes the diagonal-Q factors (unified_update_Q_factors!,
 * unified_operations.jl:468-498).                                           */
int hpr_set_sigma_lambda(hpr_ctx* ctx, double sigma, double lambda_A,
                         double lambda_Q);
int hpr_set_inner(hpr_ctx* ctx, int64_t inner);
int hpr_get_scalars(hpr_ctx* ctx, double* sigma, double* lambda_A,
                    double* lambda_Q, int64_t* inner);

/* Run k HPR iterations (main_update_gpu!, algorithm.jl:2284-2309, with
 * alpha = 1/(inner+2) and inner incremented after each iteration as in
 * perform_iteration_step!, algorithm.jl:2722-2744).  When full_last != 0 the
 * last iteration also writes x_bar, z_bar, dx, s, y_bar, dy (the "full"
 * kernels used before a residual check).                                    */
int hpr_iterate(hpr_ctx* ctx, int64_t k, int full_last);

/* KKT residuals of the current (x_bar, y_bar, z_bar[, w_bar]) in original
 * coordinates (compute_residuals!, algorithm.jl:113-196); include_bounds adds
 * the iteration-0 bound/cone violation (compute_bounds_violation!,
 * algorithm.jl:199-256).  include_bounds writes the violation into the
 * context's dx, as the reference writes ws.dx: hpr_mnorm and the restart
 * test read dx, so use include_bounds only at iteration 0 (as the solve
 * loop does) or before the next hpr_iterate with full_last != 0.            */
int hpr_compute_residuals(hpr_ctx* ctx, int include_bounds,
                          hpr_residuals* out);

/* The same residuals as hpr_compute_residuals, for callers that must not
 * allocate after set-up.  No counterpart in the reference.
 *
 * Who needs it: a host that runs its own check loop on a device whose memory
 * is already committed (for example, contexts packed up to their HBM
 * budgets), or a latency-bound loop that must never enter the CUDA allocator
 * (cudaMalloc may block; cudaFree and cudaFreeHost synchronise the whole
 * device and so stall every other stream).  This call allocates nothing: no
 * device, pinned or pageable allocation, no library routine that allocates.
 * Its reduction slots and result lanes live in a statically reserved 2 MiB
 * device array (reserved once per process and device when the library's
 * CUDA module loads), and its results go through the caller's stack.
 *
 * Limits and rules:
 *  - the problem's tile plan must fit the 2 MiB: at most 32,765 reduction
 *    slots per matrix side (one per tile of at most 704 nonzeros and 64
 *    rows, split cone and long row: about 20M nonzeros); larger problems
 *    get HPR_E_UNSUPPORTED with the sizes in hpr_last_error;
 *  - FP64 stream only (HPR_E_UNSUPPORTED after hpr_set_precision != 0);
 *  - nothing in the scratch has to start at zero: every slot is written
 *    before it is read, and nothing in the scratch carries from one call to
 *    the next (include_bounds writes the context's dx, exactly as
 *    hpr_compute_residuals does: see there);
 *  - all contexts of the process share the scratch of a device, so calls
 *    that overlapped in time would overwrite each other's partial sums; the
 *    library therefore serialises the calls per device with a host lock
 *    held until the results are back (a second caller waits);
 *  - the first call on a device looks up the scratch's device address
 *    (cudaGetSymbolAddress, which may load the module); make that first call
 *    before any stream capture.                                             */
int hpr_compute_residuals_noalloc(hpr_ctx* ctx, int include_bounds,
                                  hpr_residuals* out);

/* The context's device memory: bytes it holds within its HBM budget and the
 * number of its live device allocations (either pointer may be NULL).     */
int hpr_device_memory(hpr_ctx* ctx, size_t* used_bytes, int64_t* allocations);

/* Restart gap measure (compute_M_norm!, algorithm.jl:1302-1359), using dx,
 * dy (and dw) from the last full iteration.                                 */
int hpr_mnorm(hpr_ctx* ctx, double* out);

/* Inner products of update_sigma! (algorithm.jl:787-833):
 *   no Q : a = lambda_A*|y_bar-last_y|^2, b = |x_bar-last_x|^2, c = d = 0
 *   Q    : the a, b, c, d of the reference (diagonal Q: c = d = 0 and the
 *          sigma search over diag(Q) is hpr_sigma_golden_diag).            */
int hpr_sigma_terms(hpr_ctx* ctx, double* a, double* b, double* c, double* d);

/* Golden-section search of unified_golden_Q_diag
 * (unified_operations.jl:411-449) on the device, for diagonal Q.            */
int hpr_sigma_golden_diag(hpr_ctx* ctx, double a, double b, double lo,
                          double hi, double tol, double* sigma_out);

/* do_restart! (algorithm.jl:1130-1166): x, last_x <- x_bar; y, last_y <-
 * y_bar; with Q also w, last_w <- w_bar and ATy, last_ATy <- A'y_bar.       */
int hpr_restart(hpr_ctx* ctx);

/* Host <-> device copies of workspace vectors (HPR_VEC_*), in the scaled
 * space.  `len` must equal the vector's length.                            */
int hpr_get_vector(hpr_ctx* ctx, int which, double* host, size_t len);
int hpr_set_vector(hpr_ctx* ctx, int which, const double* host, size_t len);

/* Unscaled solution (collect_results!, algorithm.jl:1222-1256): any of the
 * pointers may be NULL.                                                     */
int hpr_get_solution(hpr_ctx* ctx, double* x, double* y, double* z, double* w);

/* Iteration schedule (no counterpart in the reference, whose iteration is
 * always a sequence of separate kernels).  Problems whose matrix sides have
 * at most 32 warp tiles can run either on the multi-CTA engine (2 launches
 * per iteration, 4 with Q) or on one CTA that runs a whole batch of
 * iterations in a single launch.  AUTO (the default) times both on the
 * first batch of a size class in the process and keeps the faster; ENGINE
 * and FUSED force one.  The iterates are identical on every schedule.      */
#define HPR_SCHEDULE_AUTO 0
#define HPR_SCHEDULE_ENGINE 1
#define HPR_SCHEDULE_FUSED 2
int hpr_set_schedule(hpr_ctx* ctx, int mode);

/* Precision of the A / A' stream (HPR_PREC_*); re-packs the scaled values.  */
int hpr_set_precision(hpr_ctx* ctx, int mode);

/* A user quadratic operator, the counterpart of a user AbstractQOperator
 * (src/Q_operators/Q_operator_interface.jl:32-151, Qmap! of
 * src/Q_operators/sparse_matrix_operator.jl:27-51): apply(user, in, out, n,
 * stream) must enqueue out = Q in on `stream` (a cudaStream_t) for device
 * vectors of length n, without synchronising the device, for a symmetric
 * positive semidefinite Q.  Call it after hpr_upload of a problem with
 * q_kind HPR_Q_NONE and before hpr_scale or a solve: the problem becomes
 * q_kind HPR_Q_OPERATOR, and, as in the reference, an operator Q turns
 * scaling off.  lambda_max_Q > 0 is used as lambda_max(Q) (a solve's
 * params.lambda_max_Q takes precedence); otherwise the power iteration
 * estimates it through `apply`.  The operator is called from the thread
 * that drives the context; it stays set until the next hpr_upload.        */
typedef void (*hpr_q_apply_fn)(void* user, const double* in, double* out, int64_t n, void* stream);
int hpr_set_q_operator(hpr_ctx* ctx, hpr_q_apply_fn apply, void* user, double lambda_max_Q);

/* The whole solve (solve(), algorithm.jl:2765-2905): scaling, power
 * iteration, the restart / sigma loop and unscaling, with the same check,
 * print and termination schedule.  `res->x/y/z/w` receive the unscaled
 * solution when non-NULL.                                                   */
int hpr_solve(hpr_ctx* ctx, const hpr_params* params, hpr_results* res);

/* Convenience: create, upload, solve, destroy in one call (optimize(),
 * algorithm.jl:2538-2581, without the JIT warm-up which has no meaning for
 * compiled kernels).                                                        */
int hpr_optimize(const hpr_problem* prob, const hpr_params* params,
                 hpr_results* res);

/* Default parameters (HPRSOCP_parameters(), src/structs.jl:277).           */
void hpr_default_params(hpr_params* p);

/* Device timing of the last hpr_iterate call's kernels, for benchmarks:
 * total device milliseconds of the x- and y-half kernels.                  */
int hpr_last_iterate_ms(hpr_ctx* ctx, double* ms_total, int64_t* launches);

/* Algorithmic bytes moved by one partial iteration (the roofline numerator
 * used by the benchmark): the plain path, or the Q path's four passes with
 * its two Q products when the problem has a Q.                             */
int hpr_iteration_bytes(hpr_ctx* ctx, double* bytes_per_iter);


/* ------------------------------------------------------------------------ */
/* Serving: continuous batching of many small problems on one device.       */
/* No single reference counterpart: it replaces calling optimize() once per */
/* model in a loop (src/algorithm.jl:2538-2581, src/utils/dataset.jl:4-122). */
/* ------------------------------------------------------------------------ */
typedef struct hpr_server hpr_server;

/* `slots` host threads on `device`, each taking requests from the queue
 * while their estimated device memory fits `hbm_budget` bytes (0 = 90% of
 * the device's free memory) and a solver context is free (four per slot).
 * A slot uploads, scales and estimates the eigenvalues of its request on
 * its context, then runs the solve loop of hpr_solve (the default), or,
 * with hpr_serve_set_resident(srv, 1), hands a problem small enough for one
 * CTA to the device-resident request loop and goes on to the next request. */
int hpr_serve_create(int device, int slots, size_t hbm_budget,
                     hpr_server** out);

/* 1: problems small enough for one CTA (every matrix side within the
 * single-CTA tile limit, FP64, no operator Q, no auto-save) are solved by
 * the device-resident request loop, a persistent kernel with one CTA per
 * solve running the whole HPR loop (iterations, residual checks, restarts,
 * sigma updates, termination) on the device; a finisher thread reads the
 * results back.  0 (default): every request runs the host loop.  The
 * device loop takes as long per iteration as the single-CTA kernel of the
 * host loop and measured lower throughput on the serving stream, so it is
 * off by default.                                                          */
int hpr_serve_set_resident(hpr_server* srv, int on);

/* Queue one problem with its own parameters (tolerance, limits, precision);
 * the problem's arrays are copied, so the caller may free them on return.
 * HPR_E_BUDGET if the request alone exceeds the server's budget.           */
int hpr_serve_submit(hpr_server* srv, const hpr_problem* prob,
                     const hpr_params* params, int64_t* ticket);

/* Wait up to wait_ms (< 0: forever) for a ticket.  HPR_OK: `res` holds the
 * result (x/y/z/w copied into the caller's buffers when non-NULL) and
 * latency_s the time from submit to completion; the ticket is consumed.
 * HPR_E_TIMEOUT: not finished yet.  HPR_E_BAD_INPUT: unknown or already
 * consumed ticket.  HPR_E_STATE: the server was stopped first.  Any other
 * code: the solve's error (message in hpr_serve_last_error).                */
int hpr_serve_poll(hpr_server* srv, int64_t ticket, int wait_ms,
                   hpr_results* res, double* latency_s);

int hpr_serve_stats(hpr_server* srv, int64_t* queued, int64_t* running,
                    size_t* reserved_bytes);

/* Time spent by the finished requests, summed: seconds[0..5] wall seconds
 * of queue wait, upload, scaling, eigenvalue estimate, solve loop, unscaled
 * read-back; seconds[6..10] the device-resident loop's seconds in
 * iterations, residual checks, M-norms, sigma updates and restarts;
 * seconds[11] its residual checks.  *requests = how many requests.        */
int hpr_serve_phase_times(hpr_server* srv, double* seconds, int64_t* requests);
const char* hpr_serve_last_error(hpr_server* srv);

/* Stops the slots after their current solves; queued requests are dropped.
 * Poll every ticket you need before destroying the server.                 */
int hpr_serve_destroy(hpr_server* srv);

/* ------------------------------------------------------------------------ */
/* CBF ingest (replaces read_cbf, src/utils/cbf_io.jl:1438-1455, with its   */
/* layout _cbf_prepare_layout, 493-634).  Host code only: no device needed. */
/* ------------------------------------------------------------------------ */
typedef struct hpr_cbf hpr_cbf; /* a parsed file; owns every array below  */

/* read_cbf's return values (the inputs of build_from_SOCP_data,
 * src/utils/builders.jl:24-108), with A as CSR instead of CSC.             */
typedef struct hpr_cbf_data {
  int64_t m;            /* rows kept: equalities, inequalities, cone rows  */
  int64_t n;            /* variables: linear ones, then cone variables     */
  int64_t number_eq;
  int64_t number_ineq;
  hpr_csr A;            /* 0-based CSR; columns ascending, no duplicates,  */
                        /* no stored zeros                                 */
  const double* rhs;    /* m: A x >= rhs / == rhs / rhs on the cone rows   */
  const double* c;      /* n (negated for OBJSENSE MAX)                    */
  const double* l;      /* n                                               */
  const double* u;      /* n                                               */
  const int64_t* soc_con_idx; /* 1-based cone row starts + end sentinel    */
  int64_t n_soc_con_idx;
  const int64_t* soc_var_idx; /* 1-based cone variable starts + sentinel   */
  int64_t n_soc_var_idx;
  double obj_constant;  /* negated for OBJSENSE MAX                        */
} hpr_cbf_data;

/* Parse a .cbf file (conic-linear subset: L+, L-, L=, F, Q) with nthreads
 * host threads (<= 0: all).  HPR_E_BAD_INPUT on a malformed or unsupported
 * file, with the reference's message in hpr_cbf_last_error().  The result
 * does not depend on nthreads.                                              */
int hpr_cbf_read(const char* path, int nthreads, hpr_cbf** out);
/* Message of this thread's last failed hpr_cbf_read ("" after a success). */
const char* hpr_cbf_last_error(void);
/* Views of the parsed arrays (valid until hpr_cbf_free).                  */
int hpr_cbf_data_get(const hpr_cbf* f, hpr_cbf_data* out);
/* The same file as a problem for hpr_upload in build_from_SOCP_data's
 * layout: AL = AU = rhs on equalities, AL = rhs / AU = +inf on
 * inequalities, soc_rhs = the cone rows' rhs, 0-based cone starts, Q = 0. */
int hpr_cbf_problem(const hpr_cbf* f, hpr_problem* out);
void hpr_cbf_free(hpr_cbf* f);

#ifdef __cplusplus
}
#endif
#endif /* HPRSOCP_B200_H */
