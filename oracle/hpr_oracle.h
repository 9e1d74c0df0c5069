/*
 * hpr_oracle.h — CPU oracle for the HPR-SOCP iteration.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain C++ FP64 restatement of the
 * reference solver's CPU path (PolyU-IOR/HPR-SOCP, Julia), used as the checker
 * for the CUDA library and as the timed CPU baseline.  Only tests/, the smoke
 * check and the benchmark's cpu_baseline / reference arm may load it; the
 * product path never does.
 *
 * Parity pins: the known-answer vectors of the reference's test/runtests.jl
 * (projection, residual, dual-objective and M-norm cases) are re-encoded in
 * tests/golden/ and checked against this oracle; the reference itself (Julia)
 * cannot run in this environment, so iterate-level parity beyond those cases
 * rests on this restatement.
 *
 * The entry points take the same structs as the product C ABI
 * (include/hprsocp_b200.h) and mirror its operations one to one, so a test can
 * drive both with identical call sequences.
 */
#ifndef HPR_ORACLE_H
#define HPR_ORACLE_H
#include "../include/hprsocp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* threads <= 0: all OpenMP threads; 1: the reference's single-threaded path */
int oracle_create(const hpr_problem* prob, int threads, oracle_ctx** out);
void oracle_destroy(oracle_ctx* o);
const char* oracle_last_error(const oracle_ctx* o);
int oracle_scale(oracle_ctx* o, const hpr_params* opts, hpr_scale_info* out);
int oracle_power_A(oracle_ctx* o, int maxit, double tol, double* lam);
int oracle_power_Q(oracle_ctx* o, int maxit, double tol, double* lam);
int oracle_set_sigma_lambda(oracle_ctx* o, double sigma, double lamA,
                            double lamQ);
int oracle_set_inner(oracle_ctx* o, int64_t inner);
int oracle_get_scalars(oracle_ctx* o, double* sigma, double* lamA,
                       double* lamQ, int64_t* inner);
int oracle_iterate(oracle_ctx* o, int64_t k, int full_last);
int oracle_residuals(oracle_ctx* o, int include_bounds, hpr_residuals* out);
int oracle_mnorm(oracle_ctx* o, double* out);
int oracle_sigma_terms(oracle_ctx* o, double* a, double* b, double* c,
                       double* d);
int oracle_sigma_golden_diag(oracle_ctx* o, double a, double b, double lo,
                             double hi, double tol, double* sigma_out);
int oracle_restart(oracle_ctx* o);
int oracle_get_vector(oracle_ctx* o, int which, double* host, size_t len);
int oracle_set_vector(oracle_ctx* o, int which, const double* host,
                      size_t len);
int oracle_get_solution(oracle_ctx* o, double* x, double* y, double* z,
                        double* w);
int oracle_solve(oracle_ctx* o, const hpr_params* params, hpr_results* res);
void oracle_default_params(hpr_params* p);

/* Scalar helpers exposed for known-answer tests of the control logic. */
double oracle_golden(double a, double b, double c, double d, double lo,
                     double hi, double tol, int maxiter);
double oracle_print_step(int64_t iter);

#ifdef __cplusplus
}
#endif
#endif
