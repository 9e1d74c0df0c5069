// hpr_serve.cpp — continuous-batching server for streams of small SOCPs.
//
// A server owns `slots` solver contexts on one device, each with its own
// CUDA stream and host thread.  Submitted requests are deep-copied into a
// FIFO; a slot takes the head of the queue as soon as it is free and the
// request's estimated device memory fits the server's HBM budget, so
// requests that arrive while others are on the GPU are admitted as slots and
// memory free up, and the kernels of all running solves overlap on the
// device (small problems launch only the CTAs their tiles need).  Each
// request carries its own parameters, so each retires at its own tolerance.
// A slot thread takes a request and a free solver context (the server keeps
// four per slot), uploads the request, scales it and estimates its
// eigenvalues.  When the problem fits one CTA (hpr_dsolve.cu), the thread
// hands its whole solve loop to the device-resident request loop (one
// persistent kernel whose CTAs each solve one request at a time, with no
// host round trip per residual check) and goes on to the next request; a
// finisher thread reads back the solutions of the requests the loop
// completes and frees their contexts.  Larger problems run the host-driven
// loop of hpr_solve on the slot thread.  Either way a request's result does
// not depend on the other requests: the same request gives the same bits
// alone and in the mix.
//
// The reference solves one model per `optimize` call (src/algorithm.jl:
// 2538-2581) and its dataset runner loops over files one at a time
// (src/utils/dataset.jl:4-122); this server is the B200 replacement for
// that loop.  It uses only the public C ABI.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "hpr_internal.h"

#ifndef HPR_SERVE_LOOP_SM_DIV
#define HPR_SERVE_LOOP_SM_DIV 3  // the request loop takes at most SMs / this many CTAs
#endif

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A request's problem with every array owned by the server.
struct OwnedCSR {
  std::vector<int32_t> rp, ci;
  std::vector<double> v;
  hpr_csr view(const hpr_csr& s) const {
    hpr_csr o = s;
    o.rowptr = s.rowptr ? rp.data() : nullptr;
    o.colind = s.colind ? ci.data() : nullptr;
    o.values = s.values ? v.data() : nullptr;
    return o;
  }
  void copy(const hpr_csr& s) {
    if (s.rowptr && s.nrows >= 0) rp.assign(s.rowptr, s.rowptr + s.nrows + 1);
    if (s.colind && s.nnz > 0) ci.assign(s.colind, s.colind + s.nnz);
    if (s.values && s.nnz > 0) v.assign(s.values, s.values + s.nnz);
  }
};

struct OwnedProblem {
  hpr_problem p{};
  OwnedCSR A, AT, Q, F;
  std::vector<double> c, l, u, AL, AU, rhs, qd;
  std::vector<int64_t> con, var;

  static void vec(std::vector<double>& dst, const double* src, int64_t n) {
    if (src && n > 0) dst.assign(src, src + n);
  }
  void copy(const hpr_problem& s) {
    p = s;
    A.copy(s.A);
    AT.copy(s.AT);
    Q.copy(s.Q);
    F.copy(s.F);
    vec(c, s.c, s.n);
    vec(l, s.l, s.n);
    vec(u, s.u, s.n);
    vec(AL, s.AL, s.m);
    vec(AU, s.AU, s.m);
    vec(rhs, s.soc_rhs, s.m - s.m_lin);
    vec(qd, s.q_diag, s.n);
    if (s.soc_con_idx && s.n_soc_con_idx > 0) con.assign(s.soc_con_idx, s.soc_con_idx + s.n_soc_con_idx);
    if (s.soc_var_idx && s.n_soc_var_idx > 0) var.assign(s.soc_var_idx, s.soc_var_idx + s.n_soc_var_idx);
    p.A = A.view(s.A);
    p.AT = AT.view(s.AT);
    p.Q = Q.view(s.Q);
    p.F = F.view(s.F);
    auto ptr = [](const std::vector<double>& v, const double* orig) { return orig ? v.data() : nullptr; };
    p.c = ptr(c, s.c);
    p.l = ptr(l, s.l);
    p.u = ptr(u, s.u);
    p.AL = ptr(AL, s.AL);
    p.AU = ptr(AU, s.AU);
    p.soc_rhs = ptr(rhs, s.soc_rhs);
    p.q_diag = ptr(qd, s.q_diag);
    p.soc_con_idx = s.soc_con_idx ? con.data() : nullptr;
    p.soc_var_idx = s.soc_var_idx ? var.data() : nullptr;
  }
};

struct Request {
  int64_t ticket = 0;
  std::unique_ptr<OwnedProblem> prob;
  hpr_params params{};
  std::string save_filename;  // owned copy of params.save_filename
  double t_submit = 0;
  size_t est = 0;
};

struct Finished {
  int rc = HPR_OK;
  std::string err;
  hpr_results res{};
  std::vector<double> x, y, z, w;
  double latency = 0;
};

// Device bytes one request needs: A and A' (value + index), the row
// pointers, ~45 workspace vectors of length n or m, reduced-precision copies,
// the tile plans and the engine's tiled copies of the matrices (values,
// indices, run padding and per-lane descriptors), with a 25% margin and
// 1 MiB of fixed overhead.
size_t estimate_bytes(const hpr_problem& p) {
  const double nnz = (double)p.A.nnz, n = (double)p.n, m = (double)p.m;
  double q = 0;
  if (p.q_kind == HPR_Q_CSR) q = (double)p.Q.nnz * 48.0;
  if (p.q_kind == HPR_Q_DIAG_LOWRANK) q = (double)p.F.nnz * 48.0 + 8.0 * n;
  const double tiles = (n + m) / 16.0 + 2.0 * nnz / 300.0 + 4.0;
  const double tiled = 2.0 * nnz * 18.0 + tiles * (144.0 + 31.0 * 18.0);
  const double b = 2.0 * nnz * (12.0 + 6.0) + 8.0 * (n + m) + 8.0 * (45.0 * n + 30.0 * m) + q + 0.05 * nnz * 32.0 +
                   tiled;
  return (size_t)(1.25 * b) + ((size_t)1 << 20);
}

}  // namespace

// A request whose solve loop is in the device-resident request loop.
struct InFlight {
  Request r;
  hpr_ctx* ctx = nullptr;
  hpr::ResidentJob job;
  Finished f;
  double ph[6] = {0, 0, 0, 0, 0, 0};
};

struct hpr_server {
  int device = 0;
  size_t budget = 0, reserved = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_flight;
  std::deque<Request> queue;
  std::map<int64_t, Finished> done;
  std::set<int64_t> live;  // submitted and not yet consumed by a poll
  std::vector<std::thread> workers;
  std::thread finisher;
  std::vector<hpr_ctx*> ctx_all, ctx_free;  // solver contexts; the free ones hold no request
  std::deque<InFlight> inflight;            // requests in the device loop
  int64_t next_ticket = 1;
  int64_t running = 0;
  int workers_alive = 0;
  bool stop = false;
  std::string err;
  hpr::DQueue* dq = nullptr;  // device-resident request loop (null: host loops only)
  int resident = 0;           // hpr_serve_set_resident
  // summed over finished requests: wall seconds of queue wait, upload,
  // scaling, eigenvalue estimate, solve loop, unscaled read-back; then the
  // device-resident loop's seconds in iterations, residual checks, M-norms,
  // sigma updates, restarts, and its residual-check count
  double phase_sum[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  int64_t phase_count = 0;

  // a request is over: record it and free its context and memory
  void complete(Request& r, Finished&& f, hpr_ctx* ctx, const double* ph) {
    f.res.x = f.res.y = f.res.z = f.res.w = nullptr;
    f.latency = now_s() - r.t_submit;
    r.prob.reset();
    {
      std::lock_guard<std::mutex> lk(mu);
      reserved -= r.est;
      --running;
      done[r.ticket] = std::move(f);
      for (int k = 0; k < 6; ++k) phase_sum[k] += ph[k];
      for (int k = 0; k < 6; ++k) phase_sum[6 + k] += ctx->c.dloop[k];
      for (int k = 0; k < 6; ++k) ctx->c.dloop[k] = 0.0;
      ++phase_count;
      ctx_free.push_back(ctx);
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }

  // A slot thread: takes the head of the queue once its memory fits and a
  // context is free, uploads it, scales it and estimates its eigenvalues,
  // then either hands the solve loop to the device (and goes on to the next
  // request) or runs the host loop to the end.
  void worker() {
    cudaSetDevice(device);
    for (;;) {
      Request r;
      hpr_ctx* ctx = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || (!queue.empty() && reserved + queue.front().est <= budget && !ctx_free.empty());
        });
        if (stop) {
          --workers_alive;
          break;
        }
        r = std::move(queue.front());
        queue.pop_front();
        reserved += r.est;
        ++running;
        ctx = ctx_free.back();
        ctx_free.pop_back();
      }
      Finished f;
      const int64_t n = r.prob->p.n, m = r.prob->p.m;
      f.x.assign((size_t)n, 0.0);
      f.y.assign((size_t)m, 0.0);
      f.z.assign((size_t)n, 0.0);
      f.w.assign((size_t)n, 0.0);
      f.res.x = f.x.data();
      f.res.y = f.y.data();
      f.res.z = f.z.data();
      f.res.w = f.w.data();
      r.params.verbose = 0;
      r.params.device_number = device;
      r.params.save_filename = r.save_filename.empty() ? nullptr : r.save_filename.c_str();
      double ph[6] = {0, 0, 0, 0, 0, 0};
      const double t_start = now_s();
      ph[0] = t_start - r.t_submit;
      f.rc = hpr_upload(ctx, &r.prob->p);
      ph[1] = now_s() - t_start;
      hpr::ResidentJob job;
      bool submitted = false;
      if (f.rc == HPR_OK)
        f.rc = hpr::solve_resident_begin(&ctx->c, &r.params, &f.res, resident ? dq : nullptr, &job, &submitted,
                                         ph + 2);
      if (f.rc != HPR_OK) f.err = hpr_last_error(ctx);
      if (f.rc == HPR_OK && submitted) {
        InFlight fl;
        fl.r = std::move(r);
        fl.ctx = ctx;
        fl.job = job;
        fl.f = std::move(f);
        std::copy(ph, ph + 6, fl.ph);
        {
          std::lock_guard<std::mutex> lk(mu);
          inflight.push_back(std::move(fl));
        }
        cv_flight.notify_one();
        continue;
      }
      complete(r, std::move(f), ctx, ph);
    }
  }

  // Completes the requests of the device loop: polls their done flags,
  // reads back the unscaled solutions and frees their contexts.  It keeps
  // the request loop running while requests wait and drains them at stop.
  void finish_loop() {
    cudaSetDevice(device);
    double t_keep = 0.0;
    int pause_us = 20;
    for (;;) {
      std::vector<InFlight> ready;
      {
        std::unique_lock<std::mutex> lk(mu);
        if (inflight.empty()) {
          // at stop, the loop ends once no slot thread can hand over more
          if (stop && workers_alive == 0) break;
          cv_flight.wait_for(lk, std::chrono::milliseconds(5));
          continue;
        }
        for (auto it = inflight.begin(); it != inflight.end();) {
          bool fin = false;
          hpr_results r{};
          const int rc = hpr::dqueue_poll(dq, &it->ctx->c, it->job.slot, &r, &fin);
          if (fin || rc != HPR_OK) {
            InFlight fl = std::move(*it);
            it = inflight.erase(it);
            if (rc != HPR_OK) {
              fl.f.rc = rc;
              fl.f.err = hpr_last_error(fl.ctx);
            } else {
              // the done result's scalars travel in f.res until the read-back
              double *x = fl.f.res.x, *y = fl.f.res.y, *z = fl.f.res.z, *w = fl.f.res.w;
              fl.f.res = r;
              fl.f.res.x = x;
              fl.f.res.y = y;
              fl.f.res.z = z;
              fl.f.res.w = w;
            }
            ready.push_back(std::move(fl));
          } else {
            ++it;
          }
        }
      }
      if (now_s() - t_keep > 2e-3) {
        t_keep = now_s();
        hpr::dqueue_keepalive(dq);
      }
      if (ready.empty()) {
        std::this_thread::sleep_for(std::chrono::microseconds(pause_us));
        pause_us = std::min(2 * pause_us, 200);
        continue;
      }
      pause_us = 20;
      for (InFlight& fl : ready) {
        const double t_back = now_s();
        fl.ph[4] = t_back - fl.job.t_loop;
        if (fl.f.rc == HPR_OK) {
          const hpr_results r = fl.f.res;
          fl.f.rc = hpr::solve_resident_end(&fl.ctx->c, fl.job, r, &fl.f.res);
          if (fl.f.rc != HPR_OK) fl.f.err = hpr_last_error(fl.ctx);
        }
        fl.ph[5] = now_s() - t_back;
        complete(fl.r, std::move(fl.f), fl.ctx, fl.ph);
      }
    }
  }
};

extern "C" {

int hpr_serve_create(int device, int slots, size_t hbm_budget, hpr_server** out) {
  if (!out || slots < 1 || slots > 1024) return HPR_E_BAD_INPUT;
  *out = nullptr;
  // The slots' streams run concurrently only if the device context has as
  // many hardware work queues; CUDA's default is 8.  This takes effect when
  // it is set before the process creates its CUDA context (an existing
  // setting is kept).
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  // Many slot threads wait on the device at once: when the server creates
  // the process's CUDA context, its waits block instead of spinning, so the
  // waiting threads leave the host cores to the threads preparing requests.
  // (An existing context keeps its own mode; the call then fails harmlessly.)
  if (cudaInitDevice(device, cudaDeviceScheduleBlockingSync, 0) != cudaSuccess) (void)cudaGetLastError();
  // up to four requests per slot thread can be in the device loop at once,
  // each on a context of its own
  const int nctx = 4 * slots;
  std::vector<hpr_ctx*> ctxs;
  for (int i = 0; i < nctx; ++i) {
    hpr_ctx* c = nullptr;
    int rc = hpr_create(device, 0, &c);
    if (rc != HPR_OK) {
      for (hpr_ctx* d : ctxs) hpr_destroy(d);
      return rc;
    }
    ctxs.push_back(c);
  }
  hpr_server* s = new hpr_server();
  s->device = device;
  if (hbm_budget == 0) {
    // 90% of what the device has free, as a single context would take
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      for (hpr_ctx* d : ctxs) hpr_destroy(d);
      delete s;
      return HPR_E_CUDA;
    }
    hbm_budget = (size_t)(0.9 * (double)fr);
  }
  s->budget = hbm_budget;
  std::string qerr;
  // one CTA of the request loop per context that can be in it, and at most
  // a third of the SMs (a loop CTA takes a whole SM's registers): the other
  // SMs stay free for the upload, scaling and eigenvalue kernels of the
  // requests being set up and for the multi-CTA engine of the requests too
  // large for one CTA
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  s->dq = hpr::dqueue_create(device, std::max(1, std::min(nctx, sms / HPR_SERVE_LOOP_SM_DIV)), 4096, &qerr);
  if (!s->dq) {
    for (hpr_ctx* d : ctxs) hpr_destroy(d);
    delete s;
    return HPR_E_CUDA;
  }
  s->ctx_all = ctxs;
  s->ctx_free = ctxs;
  s->workers_alive = slots;
  for (int i = 0; i < slots; ++i) s->workers.emplace_back([s] { s->worker(); });
  s->finisher = std::thread([s] { s->finish_loop(); });
  *out = s;
  return HPR_OK;
}

int hpr_serve_set_resident(hpr_server* s, int on) {
  if (!s) return HPR_E_BAD_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  s->resident = on ? 1 : 0;
  return HPR_OK;
}

int hpr_serve_submit(hpr_server* s, const hpr_problem* prob, const hpr_params* params, int64_t* ticket) {
  if (!s || !prob || !ticket) return HPR_E_BAD_INPUT;
  if (prob->m < 0 || prob->n < 0 || prob->A.nnz < 0) return HPR_E_BAD_INPUT;
  Request r;
  r.est = estimate_bytes(*prob);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (r.est > s->budget) {
      s->err = "request needs about " + std::to_string(r.est) + " bytes; the server's HBM budget is " +
               std::to_string(s->budget);
      return HPR_E_BUDGET;
    }
  }
  r.prob.reset(new OwnedProblem());
  r.prob->copy(*prob);
  if (params) {
    r.params = *params;
  } else {
    hpr_default_params(&r.params);
  }
  r.params.initial_x = nullptr;  // warm starts are not carried through the queue
  r.params.initial_y = nullptr;
  if (r.params.save_filename) r.save_filename = r.params.save_filename;
  r.params.save_filename = nullptr;
  r.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r.ticket = s->next_ticket++;
    *ticket = r.ticket;
    s->live.insert(r.ticket);
    s->queue.push_back(std::move(r));
  }
  s->cv_work.notify_all();
  return HPR_OK;
}

int hpr_serve_poll(hpr_server* s, int64_t ticket, int wait_ms, hpr_results* res, double* latency_s) {
  if (!s || ticket <= 0) return HPR_E_BAD_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->live.count(ticket)) {
    s->err = "unknown or already consumed ticket " + std::to_string(ticket);
    return HPR_E_BAD_INPUT;
  }
  auto ready = [&] { return s->done.count(ticket) > 0 || s->stop; };
  if (wait_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready)) {
    return HPR_E_TIMEOUT;
  }
  if (!s->done.count(ticket)) {
    s->err = "the server was stopped before this request finished";
    return HPR_E_STATE;
  }
  Finished f = std::move(s->done[ticket]);
  s->done.erase(ticket);
  s->live.erase(ticket);
  lk.unlock();
  if (latency_s) *latency_s = f.latency;
  if (f.rc != HPR_OK) {
    std::lock_guard<std::mutex> g(s->mu);
    s->err = f.err;
    return f.rc;
  }
  if (res) {
    double *x = res->x, *y = res->y, *z = res->z, *w = res->w;
    *res = f.res;
    res->x = x;
    res->y = y;
    res->z = z;
    res->w = w;
    if (x) std::memcpy(x, f.x.data(), f.x.size() * sizeof(double));
    if (y) std::memcpy(y, f.y.data(), f.y.size() * sizeof(double));
    if (z) std::memcpy(z, f.z.data(), f.z.size() * sizeof(double));
    if (w) std::memcpy(w, f.w.data(), f.w.size() * sizeof(double));
  }
  return HPR_OK;
}

int hpr_serve_stats(hpr_server* s, int64_t* queued, int64_t* running, size_t* reserved_bytes) {
  if (!s) return HPR_E_BAD_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (queued) *queued = (int64_t)s->queue.size();
  if (running) *running = s->running;
  if (reserved_bytes) *reserved_bytes = s->reserved;
  return HPR_OK;
}

int hpr_serve_phase_times(hpr_server* s, double* seconds, int64_t* requests) {
  if (!s || !seconds) return HPR_E_BAD_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  for (int k = 0; k < 12; ++k) seconds[k] = s->phase_sum[k];
  if (requests) *requests = s->phase_count;
  return HPR_OK;
}

const char* hpr_serve_last_error(hpr_server* s) { return s ? s->err.c_str() : "null server"; }

int hpr_serve_destroy(hpr_server* s) {
  if (!s) return HPR_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  s->cv_flight.notify_all();
  for (std::thread& t : s->workers) t.join();
  // requests still in the device loop finish there first
  if (s->finisher.joinable()) s->finisher.join();
  hpr::dqueue_destroy(s->dq);
  for (hpr_ctx* c : s->ctx_all) hpr_destroy(c);
  delete s;
  return HPR_OK;
}

}  // extern "C"
