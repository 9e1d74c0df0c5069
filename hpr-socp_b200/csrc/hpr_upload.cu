// hpr_upload.cu — device-side CSR ingest: validation, index-base conversion
// and transposition.
//
// The reference converts its model to GPU matrices once per solve
// (QP_info_gpu construction, src/algorithm.jl:2318-2352) and forms A' with
// CUSPARSE (transpose of the CuSparseMatrixCSR).  Here the caller's column
// and value arrays are copied to HBM unchanged and checked there, one warp
// per row: column range, finiteness of the values and ascending columns.
// The transpose is a stable radix sort of the column indices, so every row of
// A' lists its entries in ascending row order — the canonical order the CPU
// restatement builds by counting sort — and the result is deterministic.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "hpr_internal.h"

namespace hpr {

namespace {

enum : int { kBadColumn = 1, kBadValue = 2, kUnsorted = 4 };

// One warp per row: subtract the index base in place, flag out-of-range
// columns, non-finite values and descending column pairs.
__global__ void csr_check_kernel(const int32_t* __restrict__ rp, int32_t* __restrict__ col,
                                 const double* __restrict__ val, int64_t nr, int64_t nc, int base,
                                 int* __restrict__ flags) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int bad = 0;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nr; r += nwarps) {
    const int32_t b = rp[r], e = rp[r + 1];
    int64_t prev = LLONG_MIN;  // last column of the previous 32-entry chunk
    for (int32_t k0 = b; k0 < e; k0 += 32) {
      const int32_t k = k0 + lane;
      int64_t j = LLONG_MAX;
      if (k < e) {
        j = (int64_t)col[k] - base;
        if (j < 0 || j >= nc) bad |= kBadColumn;
        if (!isfinite(val[k])) bad |= kBadValue;
        col[k] = (int32_t)j;
      }
      int64_t left = __shfl_up_sync(0xffffffffu, j, 1);
      if (lane == 0) left = prev;
      if (k < e && j < left) bad |= kUnsorted;
      prev = __shfl_sync(0xffffffffu, j, 31);
    }
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  if (lane == 0 && bad) atomicOr(flags, bad);
}

__global__ void col_count_kernel(const int32_t* __restrict__ col, int64_t nnz, int32_t* __restrict__ cnt) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cnt + col[k] + 1, 1);
}

__global__ void iota_kernel(int32_t* __restrict__ v, int64_t n) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    v[k] = (int32_t)k;
}

// row index of every nonzero (one warp per row)
__global__ void row_of_kernel(const int32_t* __restrict__ rp, int64_t nr, int32_t* __restrict__ row) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nr; r += nwarps)
    for (int32_t k = rp[r] + lane; k < rp[r + 1]; k += 32) row[k] = (int32_t)r;
}

__global__ void transpose_gather_kernel(const int32_t* __restrict__ perm, const int32_t* __restrict__ row,
                                        const double* __restrict__ val, int64_t nnz, int32_t* __restrict__ tcol,
                                        double* __restrict__ tval) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t k = perm[p];
    tcol[p] = row[k];
    tval[p] = val[k];
  }
}

int grid_for(int64_t work) {
  int64_t g = (work + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// Scratch that lives only for the duration of one upload step (released in
// stream order after the work that uses it).
struct Scratch {
  Ctx* c;
  std::vector<void*> ptrs;
  explicit Scratch(Ctx* cc) : c(cc) {}
  template <class T>
  int get(T** p, int64_t n) {
    HPR_TRY(dev_alloc(c, (void**)p, (size_t)std::max<int64_t>(n, 1) * sizeof(T)));
    ptrs.push_back(*p);
    return HPR_OK;
  }
  int bytes(void** p, size_t b) {
    HPR_TRY(dev_alloc(c, p, b));
    ptrs.push_back(*p);
    return HPR_OK;
  }
  ~Scratch() {
    for (void* p : ptrs) dev_free(c, p);
  }
};

// Rows of an unsorted matrix are ordered on the host (stable in the value
// order for equal columns, as a CSC build by insertion would be).
int sort_rows_on_host(Ctx* c, DevCSR& M, const std::vector<int32_t>& rp) {
  std::vector<int32_t> ci(M.nnz);
  std::vector<double> v(M.nnz);
  HPR_CUDA(c, cudaMemcpyAsync(ci.data(), M.col, M.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA(c, cudaMemcpyAsync(v.data(), M.val, M.nnz * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  std::vector<std::pair<int32_t, double>> tmp;
  for (int64_t i = 0; i < M.nrows; ++i) {
    tmp.clear();
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) tmp.push_back({ci[k], v[k]});
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                       return a.first < b.first;
                     });
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      ci[k] = tmp[k - rp[i]].first;
      v[k] = tmp[k - rp[i]].second;
    }
  }
  HPR_CUDA(c, cudaMemcpyAsync(M.col, ci.data(), M.nnz * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  HPR_CUDA(c, cudaMemcpyAsync(M.val, v.data(), M.nnz * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

// ---- staged host-to-device copies
//
// A pageable copy is staged by the driver through its own pinned buffer at
// about 9 GB/s (measured: 300 MB of A in 33 ms on the benchmark SOCP).  Here
// kStageThreads host threads each fill their own pair of pinned chunks and
// enqueue the chunk's DMA on the context stream, so the host copies run in
// parallel and overlap the transfers.  The chunks belong to the device
// (one set per device, shared by its contexts under a mutex); an event per
// chunk tells when its previous DMA has drained.
constexpr int kStageThreads = 8;
constexpr int kStageSlots = 2;
constexpr size_t kStageChunk = (size_t)4 << 20;
constexpr size_t kStageMin = (size_t)4 << 20;  // smaller copies go straight to cudaMemcpyAsync
constexpr int kStageDevices = 64;

struct Stage {
  std::mutex mu;
  bool tried = false, ok = false;
  void* buf[kStageThreads][kStageSlots] = {};
  cudaEvent_t ev[kStageThreads][kStageSlots] = {};
  bool used[kStageThreads][kStageSlots] = {};
};
Stage g_stage[kStageDevices];

// allocates the device's chunks once (caller holds st.mu); false if the
// pinned memory or the events are not available
bool stage_init(Stage& st, int device) {
  if (st.tried) return st.ok;
  st.tried = true;
  cudaSetDevice(device);
  for (int t = 0; t < kStageThreads; ++t)
    for (int k = 0; k < kStageSlots; ++k) {
      if (cudaHostAlloc(&st.buf[t][k], kStageChunk, cudaHostAllocPortable) != cudaSuccess ||
          cudaEventCreateWithFlags(&st.ev[t][k], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    }
  st.ok = true;
  return true;
}

}  // namespace

namespace {

// every double of v[0, n) passes (check 1: finite; check 2: not NaN); the
// bit tests keep the loop branch-free
bool doubles_ok(const void* p, size_t n, int check) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  uint64_t bad = 0;
  for (size_t i = 0; i < n; ++i) {
    uint64_t w;
    std::memcpy(&w, b + 8 * i, 8);
    const uint64_t a = w & 0x7fffffffffffffffull;
    bad |= check == 1 ? (uint64_t)(a >= 0x7ff0000000000000ull) : (uint64_t)(a > 0x7ff0000000000000ull);
  }
  return bad == 0;
}

}  // namespace

int h2d_copy(Ctx* c, void* dst, const void* src, size_t bytes) { return h2d_copy_checked(c, dst, src, bytes, 0, nullptr); }

int h2d_copy_checked(Ctx* c, void* dst, const void* src, size_t bytes, int check, bool* ok) {
  if (ok) *ok = true;
  if (bytes == 0) return HPR_OK;
  if (bytes < kStageMin || c->device < 0 || c->device >= kStageDevices) {
    if (check && ok) *ok = doubles_ok(src, bytes / 8, check);
    HPR_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return HPR_OK;
  }
  Stage& st = g_stage[c->device];
  std::lock_guard<std::mutex> lock(st.mu);
  if (!stage_init(st, c->device)) {
    if (check && ok) *ok = doubles_ok(src, bytes / 8, check);
    HPR_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return HPR_OK;
  }
  const size_t nchunks = (bytes + kStageChunk - 1) / kStageChunk;
  std::atomic<int> err{0};
  std::atomic<bool> good{true};
  auto worker = [&](int t) {
    if (cudaSetDevice(c->device) != cudaSuccess) {
      err.store(1);
      return;
    }
    int use = 0;
    // thread t copies chunks t, t + kStageThreads, ... through its slots in turn
    for (size_t k = (size_t)t; k < nchunks && !err.load(); k += kStageThreads, use ^= 1) {
      const size_t off = k * kStageChunk;
      const size_t len = std::min(kStageChunk, bytes - off);
      if (st.used[t][use] && cudaEventSynchronize(st.ev[t][use]) != cudaSuccess) {
        err.store(1);
        return;
      }
      std::memcpy(st.buf[t][use], static_cast<const char*>(src) + off, len);
      // the values are checked in the pinned chunk, while it is in cache
      if (check && !doubles_ok(st.buf[t][use], len / 8, check)) good.store(false);
      if (cudaMemcpyAsync(static_cast<char*>(dst) + off, st.buf[t][use], len, cudaMemcpyHostToDevice, c->stream) !=
              cudaSuccess ||
          cudaEventRecord(st.ev[t][use], c->stream) != cudaSuccess) {
        err.store(1);
        return;
      }
      st.used[t][use] = true;
    }
  };
  const int nt = (int)std::min<size_t>(kStageThreads, nchunks);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) spawn_or_run(th, [&worker, t] { worker(t); });
  worker(0);
  for (auto& x : th) x.join();
  if (err.load()) return set_err(c, HPR_E_CUDA, "staged host-to-device copy failed");
  if (ok) *ok = good.load();
  return HPR_OK;
}

int d2h_copy(Ctx* c, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return HPR_OK;
  if (bytes < kStageMin || c->device < 0 || c->device >= kStageDevices) {
    HPR_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
    return HPR_OK;
  }
  Stage& st = g_stage[c->device];
  std::lock_guard<std::mutex> lock(st.mu);
  if (!stage_init(st, c->device)) {
    HPR_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    HPR_CUDA(c, cudaStreamSynchronize(c->stream));
    return HPR_OK;
  }
  const size_t nchunks = (bytes + kStageChunk - 1) / kStageChunk;
  std::atomic<int> err{0};
  // thread t moves chunks t, t + kStageThreads, ...: the chunk's DMA into
  // its pinned slot, then (once that DMA is done) the host copy out of it
  auto worker = [&](int t) {
    if (cudaSetDevice(c->device) != cudaSuccess) {
      err.store(1);
      return;
    }
    int use = 0;
    for (size_t k = (size_t)t; k < nchunks && !err.load(); k += kStageThreads, use ^= 1) {
      const size_t off = k * kStageChunk;
      const size_t len = std::min(kStageChunk, bytes - off);
      if (st.used[t][use] && cudaEventSynchronize(st.ev[t][use]) != cudaSuccess) {
        err.store(1);
        return;
      }
      if (cudaMemcpyAsync(st.buf[t][use], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost,
                          c->stream) != cudaSuccess ||
          cudaEventRecord(st.ev[t][use], c->stream) != cudaSuccess ||
          cudaEventSynchronize(st.ev[t][use]) != cudaSuccess) {
        err.store(1);
        return;
      }
      st.used[t][use] = true;
      std::memcpy(static_cast<char*>(dst) + off, st.buf[t][use], len);
    }
  };
  const int nt = (int)std::min<size_t>(kStageThreads, nchunks);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) spawn_or_run(th, [&worker, t] { worker(t); });
  worker(0);
  for (auto& x : th) x.join();
  if (err.load()) return set_err(c, HPR_E_CUDA, "staged device-to-host copy failed");
  return HPR_OK;
}

bool host_all(const double* v, int64_t n, bool (*pred)(double)) {
  constexpr int64_t kPar = (int64_t)1 << 20;  // shorter arrays: one thread
  if (n < kPar) {
    for (int64_t i = 0; i < n; ++i)
      if (!pred(v[i])) return false;
    return true;
  }
  const int nt = (int)std::min<int64_t>(8, std::max<int64_t>(1, std::thread::hardware_concurrency()));
  std::atomic<bool> good{true};
  auto part = [&](int t) {
    const int64_t b = n * t / nt, e = n * (t + 1) / nt;
    for (int64_t i = b; i < e; ++i)
      if (!pred(v[i])) {
        good.store(false);
        return;
      }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) spawn_or_run(th, [&part, t] { part(t); });
  part(0);
  for (auto& x : th) x.join();
  return good.load();
}

int upload_csr(Ctx* c, const hpr_csr& s, int base, int64_t nr, int64_t nc, const char* name, DevCSR& M,
               std::vector<int32_t>& rp) {
  const std::string nm(name);
  if (s.nrows != nr || s.ncols != nc) return set_err(c, HPR_E_BAD_INPUT, nm + ": dimensions do not match the problem");
  if (s.nnz < 0 || s.nnz > (int64_t)std::numeric_limits<int32_t>::max())
    return set_err(c, HPR_E_BAD_INPUT, nm + ": nnz out of range");
  if (nr > 0 && !s.rowptr) return set_err(c, HPR_E_BAD_INPUT, nm + ": null rowptr");
  if (s.nnz > 0 && (!s.colind || !s.values)) return set_err(c, HPR_E_BAD_INPUT, nm + ": null arrays");
  rp.assign(nr + 1, 0);
  if (nr == 0 && s.nnz != 0) return set_err(c, HPR_E_BAD_INPUT, nm + ": nonzeros without rows");
  if (nr > 0) {
    for (int64_t i = 0; i <= nr; ++i) rp[i] = s.rowptr[i] - base;
    if (rp[0] != 0 || rp[nr] != s.nnz) return set_err(c, HPR_E_BAD_INPUT, nm + ": rowptr does not span nnz");
    for (int64_t i = 0; i < nr; ++i)
      if (rp[i + 1] < rp[i]) return set_err(c, HPR_E_BAD_INPUT, nm + ": rowptr decreases");
  }
  M.nrows = nr;
  M.ncols = nc;
  M.nnz = s.nnz;
  HPR_TRY(dev_alloc_n(c, &M.rowptr, nr + 1));
  HPR_TRY(dev_alloc_n(c, &M.col, M.nnz));
  HPR_TRY(dev_alloc_n(c, &M.val, M.nnz));
  HPR_CUDA(c, cudaMemcpyAsync(M.rowptr, rp.data(), (nr + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  if (M.nnz == 0) return HPR_OK;
  HPR_TRY(h2d_copy(c, M.col, s.colind, M.nnz * sizeof(int32_t)));
  HPR_TRY(h2d_copy(c, M.val, s.values, M.nnz * sizeof(double)));
  int* flags = nullptr;
  Scratch sc(c);
  HPR_TRY(sc.get(&flags, 1));
  HPR_CUDA(c, cudaMemsetAsync(flags, 0, sizeof(int), c->stream));
  csr_check_kernel<<<grid_for(nr * 32), 256, 0, c->stream>>>(M.rowptr, M.col, M.val, nr, nc, base, flags);
  HPR_CUDA(c, cudaGetLastError());
  int h = 0;
  HPR_CUDA(c, cudaMemcpyAsync(&h, flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h & kBadColumn) return set_err(c, HPR_E_BAD_INPUT, nm + ": column index out of range");
  if (h & kBadValue) return set_err(c, HPR_E_BAD_INPUT, nm + ": non-finite value");
  if (h & kUnsorted) HPR_TRY(sort_rows_on_host(c, M, rp));
  return HPR_OK;
}

int transpose_csr(Ctx* c, const DevCSR& M, DevCSR& T, std::vector<int32_t>& trp) {
  const int64_t nnz = M.nnz, nr = M.nrows, nc = M.ncols;
  T.nrows = nc;
  T.ncols = nr;
  T.nnz = nnz;
  HPR_TRY(dev_alloc_n(c, &T.rowptr, nc + 1));
  HPR_TRY(dev_alloc_n(c, &T.col, nnz));
  HPR_TRY(dev_alloc_n(c, &T.val, nnz));
  HPR_CUDA(c, cudaMemsetAsync(T.rowptr, 0, (nc + 1) * sizeof(int32_t), c->stream));
  trp.assign(nc + 1, 0);
  if (nnz > 0) {
    Scratch sc(c);
    int32_t *keys_out, *perm_in, *perm_out, *row;
    HPR_TRY(sc.get(&keys_out, nnz));
    HPR_TRY(sc.get(&perm_in, nnz));
    HPR_TRY(sc.get(&perm_out, nnz));
    HPR_TRY(sc.get(&row, nnz));
    // column counts -> A' row pointers
    col_count_kernel<<<grid_for(nnz), 256, 0, c->stream>>>(M.col, nnz, T.rowptr);
    HPR_CUDA(c, cudaGetLastError());
    size_t scan_bytes = 0, sort_bytes = 0;
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < nc) ++end_bit;
    HPR_CUDA(c, cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, T.rowptr + 1, T.rowptr + 1, (int)nc, c->stream));
    HPR_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, M.col, keys_out, perm_in, perm_out, (int)nnz, 0,
                                                end_bit, c->stream));
    void* tmp = nullptr;
    const size_t tmp_bytes = std::max(scan_bytes, sort_bytes);
    HPR_TRY(sc.bytes(&tmp, tmp_bytes));
    size_t b1 = tmp_bytes, b2 = tmp_bytes;
    HPR_CUDA(c, cub::DeviceScan::InclusiveSum(tmp, b1, T.rowptr + 1, T.rowptr + 1, (int)nc, c->stream));
    // stable sort of the column indices: equal columns keep ascending rows
    iota_kernel<<<grid_for(nnz), 256, 0, c->stream>>>(perm_in, nnz);
    HPR_CUDA(c, cudaGetLastError());
    HPR_CUDA(c, cub::DeviceRadixSort::SortPairs(tmp, b2, M.col, keys_out, perm_in, perm_out, (int)nnz, 0, end_bit,
                                                c->stream));
    row_of_kernel<<<grid_for(nr * 32), 256, 0, c->stream>>>(M.rowptr, nr, row);
    HPR_CUDA(c, cudaGetLastError());
    transpose_gather_kernel<<<grid_for(nnz), 256, 0, c->stream>>>(perm_out, row, M.val, nnz, T.col, T.val);
    HPR_CUDA(c, cudaGetLastError());
  }
  HPR_CUDA(c, cudaMemcpyAsync(trp.data(), T.rowptr, (nc + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  HPR_CUDA(c, cudaStreamSynchronize(c->stream));
  return HPR_OK;
}

}  // namespace hpr
