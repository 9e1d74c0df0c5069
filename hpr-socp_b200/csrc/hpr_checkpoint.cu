// hpr_checkpoint.cu — auto-save of the current and best iterates.
//
// The reference keeps the best iterate seen at a residual check
// (compute_residuals!, src/algorithm.jl:176-195: saved when iter == 0 or
// when the KKT measure beats max(save_err_Rp, save_err_Rd, save_rel_gap))
// and, with `auto_save`, writes the current and best iterates in original
// coordinates plus the parameters to a file on every print iteration and at
// termination (src/algorithm.jl:2871-2880, save_state_to_hdf5! 306-421).
//
// Here the loop never waits for that file:
//   * the best iterate is a device-to-device copy of x_bar, y_bar, z_bar
//     (and w_bar) on the solver stream, taken after the residual check;
//   * a save unscales the current and the best iterates into a device
//     staging area (one map kernel per vector), and a second stream copies
//     the staging area to pinned host memory while the solver stream runs
//     on;
//   * a writer thread waits for that copy and writes the archive to a
//     temporary file beside it, then renames it over `save_filename`, so a
//     reader never sees a half-written file.
// A print iteration that comes while the previous file is still being
// written is not saved, so auto-save never holds the iteration back (the
// reference writes every print iteration, synchronously); the final
// iteration is always saved, and the call that started the solve returns
// after its file is complete.  The solver stream waits (on the device) for
// the previous copy before it overwrites the staging area.  The CRC-32 of
// the archive's vectors are computed on one thread each.
//
// The file is a NumPy .npz archive (hpr_npz.h) with the reference's HDF5
// paths as member names: no HDF5 library is available to this build.
#include "hpr_engine.cuh"
#include "hpr_internal.h"
#include "hpr_npz.h"

#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <ctime>
#include <mutex>
#include <thread>

namespace hpr {

namespace {

const char* bc_norm_name(int k) {
  switch (k) {
    case HPR_BC_NORM_L2: return "l2";
    case HPR_BC_NORM_RMS: return "rms";
    case HPR_BC_NORM_LINF: return "linf";
    default: return "unknown";
  }
}

const char* soc_strategy_name(int k) {
  static const char* names[] = {"",
                                "max",
                                "rms",
                                "geom",
                                "adaptive",
                                "hybrid",
                                "ruiz_geom",
                                "role_split",
                                "pock_safe_role_split",
                                "size_split_role_split",
                                "pre_pock_size_split",
                                "pre_pock_huge_var_taper",
                                "pre_pock_huge_var_taper_pock_geom",
                                "pre_pock_band_split",
                                "pre_pock_constraint_rms",
                                "pre_pock_constraint_max",
                                "pre_pock_constraint_taper",
                                "small_cone_constraint_max",
                                "count_aware_small_cone_bias",
                                "phase_blend",
                                "phase_taper"};
  return (k >= 1 && k <= 20) ? names[k] : "unknown";
}

// local time as yyyy-mm-ddTHH:MM:SS.sss
std::string timestamp_now() {
  using namespace std::chrono;
  const auto now = system_clock::now();
  const std::time_t t = system_clock::to_time_t(now);
  const int ms = (int)(duration_cast<milliseconds>(now.time_since_epoch()).count() % 1000);
  std::tm tmv{};
  localtime_r(&t, &tmv);
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%04d-%02d-%02dT%02d:%02d:%02d.%03d", tmv.tm_year + 1900, tmv.tm_mon + 1,
                tmv.tm_mday, tmv.tm_hour, tmv.tm_min, tmv.tm_sec, ms);
  return buf;
}

}  // namespace

struct Checkpointer {
  struct Best {
    int64_t iter = 0;
    double sigma = 0.0;
    hpr_residuals rs{};
  };
  struct Job {
    int64_t iter = 0;
    double elapsed = 0.0, sigma = 0.0;
    std::string stamp;
    hpr_residuals rs{};
    Best best;
  };

  Ctx* c;
  hpr_params P;
  std::string path;
  int64_t n = 0, m = 0;
  bool has_q = false;
  // best iterate, scaled (w only with a quadratic term)
  double *sx = nullptr, *sy = nullptr, *sz = nullptr, *sw = nullptr;
  bool have_best = false;
  Best best;
  // staging: current x, w, z, y then best x, w, z, y (w only with Q)
  double* stage = nullptr;
  double* host = nullptr;
  int64_t stage_len = 0;
  cudaStream_t copy = nullptr;
  cudaEvent_t staged = nullptr, copied = nullptr;
  bool copy_pending = false;
  // writer thread
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  bool has_job = false, busy = false, stop = false;
  Job job;
  std::string write_err;
  int64_t files = 0, skipped = 0;

  Checkpointer(Ctx* ctx, const hpr_params* p) : c(ctx), P(*p) {
    path = (p->save_filename && p->save_filename[0]) ? p->save_filename : "HPRSOCP_autosave.npz";
  }

  int64_t vec_len() const { return (has_q ? 3 : 2) * n + m; }  // one iterate in the staging area

  int init() {
    n = c->n;
    m = c->m;
    has_q = c->has_q;
    HPR_TRY(dev_alloc_n(c, &sx, n));
    HPR_TRY(dev_alloc_n(c, &sz, n));
    HPR_TRY(dev_alloc_n(c, &sy, m));
    if (has_q) HPR_TRY(dev_alloc_n(c, &sw, n));
    stage_len = 2 * vec_len();
    HPR_TRY(dev_alloc_n(c, &stage, stage_len));
    HPR_CUDA(c, cudaMallocHost((void**)&host, (size_t)(stage_len > 0 ? stage_len : 1) * sizeof(double)));
    HPR_CUDA(c, cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
    HPR_CUDA(c, cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    HPR_CUDA(c, cudaEventCreateWithFlags(&copied, cudaEventDisableTiming | cudaEventBlockingSync));
    th = std::thread([this] { writer_main(); });
    return HPR_OK;
  }

  // compute_residuals! best-iterate bookkeeping (algorithm.jl:176-195)
  int track(int64_t iter, double sigma, const hpr_residuals& rs) {
    const double saved = std::max(std::max(best.rs.err_Rp_org_bar, best.rs.err_Rd_org_bar), best.rs.rel_gap_bar);
    if (!(iter == 0 || !have_best || rs.KKTx_and_gap_org_bar < saved)) return HPR_OK;
    const size_t nb = (size_t)n * sizeof(double), mb = (size_t)m * sizeof(double);
    HPR_CUDA(c, cudaMemcpyAsync(sx, c->x_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
    HPR_CUDA(c, cudaMemcpyAsync(sz, c->z_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
    if (m > 0) HPR_CUDA(c, cudaMemcpyAsync(sy, c->y_bar, mb, cudaMemcpyDeviceToDevice, c->stream));
    if (has_q) HPR_CUDA(c, cudaMemcpyAsync(sw, c->w_bar, nb, cudaMemcpyDeviceToDevice, c->stream));
    have_best = true;
    best.iter = iter;
    best.sigma = sigma;
    best.rs = rs;
    return HPR_OK;
  }

  // original coordinates (algorithm.jl:95-102): x = b_s x/col, y = c_s y/row,
  // z = c_s z.*col, into stage[off ...]
  int unscale_into(int64_t off, const double* xb, const double* wb, const double* zb, const double* yb) {
    const double bs = c->b_scale, cs = c->c_scale;
    const double *col = c->col_norm, *row = c->row_norm;
    double* t = stage + off;
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { t[i] = bs * (xb[i] / col[i]); }));
    t += n;
    if (has_q) {
      HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { t[i] = bs * (wb[i] / col[i]); }));
      t += n;
    }
    HPR_TRY(vec_map(c, n, [=] __device__(int64_t i) { t[i] = cs * (zb[i] * col[i]); }));
    t += n;
    HPR_TRY(vec_map(c, m, [=] __device__(int64_t i) { t[i] = cs * (yb[i] / row[i]); }));
    return HPR_OK;
  }

  int save(int64_t iter, double elapsed, double sigma, const hpr_residuals& rs, bool final) {
    {
      std::unique_lock<std::mutex> lk(mu);
      if (!final && (busy || has_job)) {
        ++skipped;  // the writer is behind: this print iteration is not saved
        return HPR_OK;
      }
      cv.wait(lk, [this] { return !busy && !has_job; });
    }
    if (copy_pending) HPR_CUDA(c, cudaStreamWaitEvent(c->stream, copied, 0));
    HPR_TRY(unscale_into(0, c->x_bar, c->w_bar, c->z_bar, c->y_bar));
    HPR_TRY(unscale_into(vec_len(), sx, sw, sz, sy));
    HPR_CUDA(c, cudaEventRecord(staged, c->stream));
    HPR_CUDA(c, cudaStreamWaitEvent(copy, staged, 0));
    HPR_CUDA(c, cudaMemcpyAsync(host, stage, (size_t)stage_len * sizeof(double), cudaMemcpyDeviceToHost, copy));
    HPR_CUDA(c, cudaEventRecord(copied, copy));
    copy_pending = true;
    Job j;
    j.iter = iter;
    j.elapsed = elapsed;
    j.sigma = sigma;
    j.stamp = timestamp_now();
    j.rs = rs;
    j.best = best;
    {
      std::lock_guard<std::mutex> lk(mu);
      job = j;
      has_job = true;
    }
    cv.notify_all();
    return HPR_OK;
  }

  // Waits for the last file; a failed write is a warning, as in the
  // reference (algorithm.jl:2873-2879), not an error of the solve.
  void finish() {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [this] { return !busy && !has_job; });
    if (!write_err.empty() && P.verbose)
      std::printf("Warning: Failed to save to %s: %s\n", path.c_str(), write_err.c_str());
  }

  void writer_main() {
    cudaSetDevice(c->device);
    while (true) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [this] { return stop || has_job; });
        if (!has_job) return;
        j = job;
        has_job = false;
        busy = true;
      }
      std::string err;
      const cudaError_t e = cudaEventSynchronize(copied);
      if (e != cudaSuccess) err = std::string("device copy failed: ") + cudaGetErrorString(e);
      else err = write_file(j);
      {
        std::lock_guard<std::mutex> lk(mu);
        busy = false;
        if (!err.empty()) write_err = err;
        else ++files;
      }
      cv.notify_all();
      if (err.empty() && P.verbose) std::printf("State saved to %s at iteration %lld\n", path.c_str(), (long long)j.iter);
    }
  }

  // one archive with the reference's layout (algorithm.jl:356-418)
  std::string write_file(const Job& j) {
    // a name of its own, so solves that share save_filename (for example in
    // a server) never write the same temporary file
    static std::atomic<uint64_t> seq{0};
    const std::string tmp = path + ".tmp" + std::to_string((long long)getpid()) + "." + std::to_string(seq++);
    NpzWriter w;
    if (!w.open(tmp)) return w.error();
    const double* cur = host;
    const double* bst = host + vec_len();
    // CRC-32 of the vector members, one thread each
    struct Vec {
      const double* p;
      int64_t n;
      uint32_t crc;
    };
    std::vector<Vec> vecs;
    auto group = [&](const double* v) {
      const double* z = v + (has_q ? 2 : 1) * n;
      vecs.push_back({v, n, 0});                  // x
      vecs.push_back({has_q ? v + n : v, n, 0});  // w
      vecs.push_back({z + n, m, 0});              // y
      vecs.push_back({z, n, 0});                  // z
    };
    group(cur);
    group(bst);
    if (P.initial_x) vecs.push_back({P.initial_x, n, 0});
    if (P.initial_y) vecs.push_back({P.initial_y, m, 0});
    {
      std::vector<std::thread> crc_threads;
      for (Vec& v : vecs)
        crc_threads.emplace_back([&v] {
          v.crc = NpzWriter::member_crc("<f8", {v.n}, v.p, (size_t)v.n * sizeof(double));
        });
      for (auto& t : crc_threads) t.join();
    }
    auto vectors = [&](const char* grp, size_t first) {
      const std::string g = grp;
      const Vec* v = vecs.data() + first;
      bool ok = w.add_vector(g + "/x_org", v[0].p, n, &v[0].crc) && w.add_vector(g + "/w_org", v[1].p, n, &v[1].crc);
      if (ok && m > 0) ok = w.add_vector(g + "/y_org", v[2].p, m, &v[2].crc);
      return ok && w.add_vector(g + "/z_org", v[3].p, n, &v[3].crc);
    };
    const hpr_residuals& r = j.rs;
    const hpr_residuals& b = j.best.rs;
    bool ok = w.add_i64("current/iteration", j.iter) && w.add_f64("current/time_elapsed", j.elapsed) &&
              w.add_string("current/timestamp", j.stamp) && vectors("current", 0) &&
              w.add_f64("current/sigma", j.sigma) && w.add_f64("current/err_Rp", r.err_Rp_org_bar) &&
              w.add_f64("current/err_Rd", r.err_Rd_org_bar) && w.add_f64("current/primal_obj", r.primal_obj_bar) &&
              w.add_f64("current/dual_obj", r.dual_obj_bar) && w.add_f64("current/rel_gap", r.rel_gap_bar) &&
              w.add_f64("current/KKTx_and_gap", r.KKTx_and_gap_org_bar) && vectors("best", 4) &&
              w.add_f64("best/sigma", j.best.sigma) && w.add_i64("best/iteration", j.best.iter) &&
              w.add_f64("best/err_Rp", b.err_Rp_org_bar) && w.add_f64("best/err_Rd", b.err_Rd_org_bar) &&
              w.add_f64("best/primal_obj", b.primal_obj_bar) && w.add_f64("best/dual_obj", b.dual_obj_bar) &&
              w.add_f64("best/rel_gap", b.rel_gap_bar) &&
              w.add_f64("best/KKTx_and_gap",
                        std::max(std::max(b.err_Rp_org_bar, b.err_Rd_org_bar), b.rel_gap_bar)) &&
              w.add_f64("parameters/stoptol", P.stoptol) && w.add_f64("parameters/sigma", P.sigma) &&
              w.add_i64("parameters/max_iter", P.max_iter) && w.add_f64("parameters/time_limit", P.time_limit) &&
              w.add_i64("parameters/check_iter", P.check_iter) && w.add_bool("parameters/warm_up", false) &&
              w.add_i64("parameters/print_frequency", P.print_frequency) &&
              w.add_i64("parameters/device_number", P.device_number) &&
              w.add_bool("parameters/use_Ruiz_scaling", P.use_Ruiz_scaling != 0) &&
              w.add_i64("parameters/ruiz_iterations", P.ruiz_iterations) &&
              w.add_bool("parameters/use_bc_scaling", P.use_bc_scaling != 0) &&
              w.add_string("parameters/bc_scaling_norm_type", bc_norm_name(P.bc_scaling_norm_type)) &&
              w.add_bool("parameters/use_l2_scaling", false) &&
              w.add_bool("parameters/use_Pock_Chambolle_scaling", P.use_Pock_Chambolle_scaling != 0) &&
              w.add_string("parameters/soc_block_scaling_strategy", soc_strategy_name(P.soc_block_scaling_strategy)) &&
              w.add_bool("parameters/auto_save", true);
    if (ok && P.initial_x) ok = w.add_vector("parameters/initial_x", P.initial_x, n, &vecs[8].crc);
    if (ok && P.initial_y) ok = w.add_vector("parameters/initial_y", P.initial_y, m, &vecs[P.initial_x ? 9 : 8].crc);
    if (!w.close() || !ok) {
      std::remove(tmp.c_str());
      return w.error().empty() ? std::string("write failed") : w.error();
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
      std::remove(tmp.c_str());
      return "cannot rename " + tmp + " to " + path;
    }
    return std::string();
  }

  ~Checkpointer() {
    if (th.joinable()) {
      {
        std::lock_guard<std::mutex> lk(mu);
        stop = true;
      }
      cv.notify_all();
      // a pending job is written before the thread stops
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [this] { return !busy && !has_job; });
      }
      th.join();
    }
    if (copy_pending && copied) cudaEventSynchronize(copied);
    if (staged) cudaEventDestroy(staged);
    if (copied) cudaEventDestroy(copied);
    if (copy) cudaStreamDestroy(copy);
    if (host) cudaFreeHost(host);
    dev_free(c, stage);
    dev_free(c, sx);
    dev_free(c, sy);
    dev_free(c, sz);
    dev_free(c, sw);
  }
};

Checkpointer* ckpt_create(Ctx* c, const hpr_params* P, int* rc) {
  Checkpointer* k = new Checkpointer(c, P);
  *rc = k->init();
  if (*rc != HPR_OK) {
    delete k;
    return nullptr;
  }
  return k;
}
int ckpt_track(Checkpointer* k, int64_t iter, double sigma, const hpr_residuals& rs) {
  return k->track(iter, sigma, rs);
}
int ckpt_save(Checkpointer* k, int64_t iter, double elapsed, double sigma, const hpr_residuals& rs, bool final) {
  return k->save(iter, elapsed, sigma, rs, final);
}
void ckpt_finish(Checkpointer* k) { k->finish(); }
void ckpt_destroy(Checkpointer* k) { delete k; }

}  // namespace hpr
