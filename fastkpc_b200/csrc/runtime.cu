// Batched CI-test engine (host orchestration of the device pipeline).
//
// A batch of tests (x, y, S) becomes:
//   * designs     -- one per distinct non-empty S (host set-up, cached);
//   * components  -- one per distinct (target, S): a residual column of the
//                    device slab (|S| = 0 columns are copied, not fitted);
//   * pairs       -- one per test: (component of x, component of y).
// The device work of a batch is a fixed launch sequence on one stream:
//   gather direct columns -> fit (single / multi) -> method statistics
//   [-> guard select -> low-rank eigen -> low-rank pairs for dcc.gamma],
// captured once as a CUDA graph and replayed by execute().
#include "runtime.h"
#include "hostla.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <exception>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>

#include <unistd.h>

namespace fkpc {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(FKPC_STATUS_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

__global__ void gather_columns_kernel(const double* __restrict__ data, int n, const int* __restrict__ cols,
                                      const int* __restrict__ slots, int count, double* __restrict__ slab) {
  const int c = blockIdx.y;
  if (c >= count) return;
  const double* src = data + static_cast<int64_t>(n) * cols[c];
  double* dst = slab + static_cast<int64_t>(n) * slots[c];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

template <class T>
double upload(DevBuf<T>& buf, const std::vector<T>& host, cudaStream_t s) {
  T* d = buf.ensure(host.size());
  if (!host.empty()) cuda_check(cudaMemcpyAsync(d, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
  return static_cast<double>(host.size() * sizeof(T));
}

constexpr double kGuardLower = 0.05;
constexpr double kGuardUpper = 0.15;

}  // namespace

Engine::Engine(int device) : device_(device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) throw Error(FKPC_STATUS_NO_DEVICE, "no CUDA device is available");
  if (device < 0 || device >= count) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "CUDA device ordinal out of range");
  cuda_check(cudaSetDevice(device), "cudaSetDevice");
  cuda_check(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device), "device attribute");
  // The main stream carries the critical path (the fits, then the
  // speculative continuation, whose CTAs each need a whole SM's shared
  // memory); the side stream's statistic CTAs fill whatever it leaves, so
  // the main stream gets the highest priority and the side stream the lowest.
  int least = 0, greatest = 0;
  cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
  cuda_check(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
  cuda_check(cudaStreamCreateWithPriority(&side_, cudaStreamNonBlocking, least), "cudaStreamCreate");
  for (auto& ev : ev_) cuda_check(cudaEventCreate(&ev), "cudaEventCreate");
  cuda_check(cudaEventCreateWithFlags(&ev_warp_, cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaEventCreateWithFlags(&ev_side_, cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaEventCreateWithFlags(&ev_part_, cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaEventCreate(&ev_call_), "cudaEventCreate");
}

Engine::~Engine() {
  cudaSetDevice(device_);
  release_graph();
  if (h_arena_) cudaFreeHost(h_arena_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (h_stage_) cudaFreeHost(h_stage_);
  for (char* b : h_stage_retired_) cudaFreeHost(b);
  for (auto& ev : ev_)
    if (ev) cudaEventDestroy(ev);
  if (ev_warp_) cudaEventDestroy(ev_warp_);
  if (ev_side_) cudaEventDestroy(ev_side_);
  if (ev_part_) cudaEventDestroy(ev_part_);
  if (ev_call_) cudaEventDestroy(ev_call_);
  if (side_) {
    cudaStreamSynchronize(side_);
    cudaStreamDestroy(side_);
  }
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void Engine::stage_reset() {
  for (char* b : h_stage_retired_) cudaFreeHost(b);
  h_stage_retired_.clear();
  h_stage_used_ = 0;
}

void* Engine::stage_alloc(size_t bytes) {
  bytes = (bytes + 255) / 256 * 256;
  if (h_stage_used_ + bytes > h_stage_cap_) {
    if (h_stage_) h_stage_retired_.push_back(h_stage_);  // copies or the host may still read it
    h_stage_ = nullptr;
    const size_t cap = std::max<size_t>(2 * h_stage_cap_, 2 * bytes);
    h_stage_cap_ = 0;
    h_stage_used_ = 0;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&h_stage_), cap, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      h_stage_ = nullptr;
      throw Error(FKPC_STATUS_ALLOCATION, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
    }
    h_stage_cap_ = cap;
  }
  void* p = h_stage_ + h_stage_used_;
  h_stage_used_ += bytes;
  return p;
}

template <class T>
double Engine::stage_upload(DevBuf<T>& buf, const std::vector<T>& host, cudaStream_t st) {
  T* d = buf.ensure(host.size());
  if (host.empty()) return 0.0;
  const size_t bytes = host.size() * sizeof(T);
  void* h = stage_alloc(bytes);
  std::memcpy(h, host.data(), bytes);
  cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st ? st : stream_), "upload");
  return static_cast<double>(bytes);
}

double* Engine::pinned_arena(size_t count) {
  if (count == 0) count = 1;
  if (count > h_arena_cap_) {
    cuda_check(cudaStreamSynchronize(stream_), "arena staging");  // no copy may still read the old buffer
    if (h_arena_) cudaFreeHost(h_arena_);
    h_arena_ = nullptr;
    h_arena_cap_ = 0;
    const size_t grow = count + count / 4;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&h_arena_), grow * sizeof(double), cudaHostAllocDefault);
    if (e != cudaSuccess) {
      h_arena_ = nullptr;
      throw Error(FKPC_STATUS_ALLOCATION, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
    }
    h_arena_cap_ = grow;
  }
  return h_arena_;
}

void Engine::release_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
}

void Engine::load(const double* data, int n, int p) {
  if (n <= 5 || p < 2) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "data must have n > 5 rows and p >= 2 columns");
  for (size_t i = 0; i < static_cast<size_t>(n) * p; ++i)
    if (!std::isfinite(data[i])) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "data must contain finite doubles");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  n_ = n;
  p_ = p;
  ++load_id_;
  host_data_.assign(data, data + static_cast<size_t>(n) * p);
  double* d = d_data_.ensure(host_data_.size());
  cuda_check(cudaMemcpyAsync(d, host_data_.data(), host_data_.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
             "upload data");
  cuda_check(cudaStreamSynchronize(stream_), "upload data");
  cache_.reset(new DesignCache(host_data_.data(), n, p));
  // the cache's bivariate bases go; their device chunks are kept for reuse
  for (auto& chunk : smooth_store_) smooth_spare_.push_back(std::move(chunk));
  smooth_store_.clear();
  release_graph();
}

void Engine::plan_components(const std::vector<Test>& tests) {
  tests_ = tests;
  sets_.clear();
  comps_.clear();
  pairs_.clear();
  struct SetHash {
    size_t operator()(const std::vector<int>& v) const {
      uint64_t h = 1469598103934665603ull;  // FNV-1a over the indices
      for (int x : v) h = (h ^ static_cast<uint32_t>(x)) * 1099511628211ull;
      return static_cast<size_t>(h);
    }
  };
  std::unordered_map<std::vector<int>, int, SetHash> set_index;
  std::unordered_map<uint64_t, int> comp_index;  // (target, set or -1)
  set_index.reserve(tests.size());
  comp_index.reserve(2 * tests.size());
  const bool share = opt_.mode != FKPC_MODE_PLAIN;  // the plain form fits every test on its own
  auto component = [&](int target, int set) {
    const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(target)) << 32) | static_cast<uint32_t>(set);
    auto it = comp_index.find(key);
    if (share && it != comp_index.end()) return it->second;
    const int id = static_cast<int>(comps_.size());
    comps_.push_back(Component{target, set});
    comp_index[key] = id;
    return id;
  };
  for (size_t t = 0; t < tests_.size(); ++t) {
    Test& ts = tests_[t];
    if (ts.x < 0 || ts.x >= p_ || ts.y < 0 || ts.y >= p_ || ts.x == ts.y)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "test variables out of range");
    std::sort(ts.S.begin(), ts.S.end());
    for (size_t i = 0; i < ts.S.size(); ++i) {
      if (ts.S[i] < 0 || ts.S[i] >= p_ || ts.S[i] == ts.x || ts.S[i] == ts.y || (i > 0 && ts.S[i] == ts.S[i - 1]))
        throw Error(FKPC_STATUS_INVALID_ARGUMENT, "conditioning set must hold distinct variables other than x and y");
    }
    if (static_cast<int>(ts.S.size()) > kMaxPenalties)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "conditioning sets larger than 62 are not supported");
    int set = -1;
    if (!ts.S.empty()) {
      auto it = set_index.find(ts.S);
      if (it == set_index.end()) {
        set = static_cast<int>(sets_.size());
        sets_.push_back(ts.S);
        set_index[ts.S] = set;
      } else {
        set = it->second;
      }
    }
    PairJob job;
    job.left = component(ts.x, set);
    // a regression batch fits the targets alone: its tests' partners are
    // placeholders, given the target's component
    job.right = regress_only_ ? job.left : component(ts.y, set);
    job.out = static_cast<int>(t);
    job.pad = 0;
    pairs_.push_back(job);
  }
}

namespace {

// f(i) for i in [0, count) on up to 16 host threads.
// Host worker threads kept for the life of the process: a call's host
// set-up runs several parallel loops, and starting and joining up to 16
// threads for each cost more than the short loops themselves.  One job at a
// time: a parallel_for that finds the pool busy (another device's engine, or
// a loop nested in a job), or runs in a child forked from the process that
// started the pool (whose threads the child does not have), starts its own
// threads instead.  The pool is never destroyed: its threads wait on it until
// the process ends.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool* pool = new HostPool();
    return *pool;
  }
  // runs work() on every pool thread and on the caller; false when busy
  bool run(const std::function<void()>& work) {
    if (getpid() != owner_) return false;
    std::unique_lock<std::mutex> busy(submit_, std::try_to_lock);
    if (!busy.owns_lock() || threads_.empty()) return false;
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &work;
      pending_ = threads_.size();
      ++generation_;
    }
    wake_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
    return true;
  }

 private:
  HostPool() : owner_(getpid()) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned n = std::min(hw, 16u) - 1;
    for (unsigned w = 0; w < n; ++w) threads_.emplace_back([this] { loop(); });
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void()>* job;
      {
        std::unique_lock<std::mutex> lk(m_);
        wake_.wait(lk, [&] { return generation_ != seen; });
        seen = generation_;
        job = job_;
      }
      (*job)();
      std::lock_guard<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex submit_, m_;
  std::condition_variable wake_, done_;
  const std::function<void()>* job_ = nullptr;
  size_t pending_ = 0;
  uint64_t generation_ = 0;
  const pid_t owner_;
};

// f(i) for every i < count on the host threads; the first exception any f
// throws is rethrown to the caller once every thread has left the loop.
template <class F>
void parallel_for(size_t count, F f) {
  std::atomic<size_t> next(0);
  std::mutex error_mu;
  std::exception_ptr error;
  const std::function<void()> work = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= count) return;
      try {
        f(i);
      } catch (...) {
        std::lock_guard<std::mutex> lk(error_mu);
        if (!error) error = std::current_exception();
        next.store(count);  // the rest is skipped
      }
    }
  };
  if (count <= 1) {
    work();
  } else if (!HostPool::get().run(work)) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t workers = std::min<size_t>(std::min<size_t>(hw, 16), count);
    std::vector<std::thread> pool;
    for (size_t w = 1; w < workers; ++w) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
  }
  if (error) std::rethrow_exception(error);
}

constexpr int kTprsK = 30;                  // basis dimension of the bivariate thin-plate smooth
// Lanczos steps on the device.  The host solver, checking every 5 steps,
// converges within 60-70 steps on the 587 bivariate designs of a 500 x 50
// level; a design that has not converged by kTprsSteps is rebuilt on the host.
constexpr int kTprsSteps = kTprsK + 50;
// The univariate smooths (k = 10): the host solver converges within 25-30
// steps on a 500 x 50 level's variables.
constexpr int kTprsUniSteps = kTprsUniK + 30;
// Every bivariate design the engine builds takes the device Lanczos, however
// few there are: the per-design computation is deterministic, so a design
// comes out bit-identical whatever batch (plain or batched form) it is in.
constexpr size_t kDeviceTprsMin = 1;

}  // namespace

// The thin-plate smooths of a level that the cache lacks -- univariate
// (k = 10) and bivariate (k = 30) -- set up on the device: prepare on the
// host; Lanczos, Ritz pairs and the rest of the basis on the device; the
// basis stays there.  launch_tprs_batch enqueues the kernels and the copies of
// the penalties and column norms into page-locked memory and returns at once;
// finish_tprs_batch waits for them and puts the smooths into the cache.
// Smooths whose Ritz pairs do not converge in the batch's steps, or with too
// few unique locations, are left to the host set-up.
void Engine::launch_tprs_batch(const std::vector<std::vector<int>>& sets, int dim, TprsBatch* batch, cudaStream_t st,
                               int ctas_per_sm) {
  batch->idx.clear();
  if (sets.empty()) return;
  const int n = n_;
  const int kk = dim == 2 ? kTprsK : kTprsUniK;
  const int steps = dim == 2 ? kTprsSteps : kTprsUniSteps;
  TprsBuffers& tb = tprs_buf_[dim - 1];
  batch->dim = dim;
  const size_t count = sets.size();
  batch->sets = sets;
  batch->preps.assign(count, TprsPrep());
  batch->idx.clear();
  std::vector<char> ok(count, 0);
  parallel_for(count, [&](size_t i) {
    try {
      std::vector<double> cols(static_cast<size_t>(dim) * n);
      for (int c = 0; c < dim; ++c)
        std::copy(host_data_.begin() + static_cast<size_t>(n) * sets[i][c],
                  host_data_.begin() + static_cast<size_t>(n) * (sets[i][c] + 1),
                  cols.begin() + static_cast<size_t>(n) * c);
      batch->preps[i] = tprs_prepare(cols.data(), n, dim, kk);
      ok[i] = batch->preps[i].nu > steps && batch->preps[i].nu <= kTprsMaxNu;
    } catch (const std::exception&) {
      ok[i] = 0;  // the host set-up reports the error
    }
  });
  for (size_t i = 0; i < count; ++i)
    if (ok[i]) batch->idx.push_back(i);
  if (batch->idx.empty()) return;
  // bivariate designs the block Lanczos takes come first, the single-vector
  // runs after them; the choice depends on the design's own locations only
  auto blockable = [&](size_t i) {
    const int nu = batch->preps[i].nu;
    return dim == 2 && nu >= kTprsBlockMinNu && tprs_ld(nu) <= kTprsBlockMaxLd;
  };
  std::stable_partition(batch->idx.begin(), batch->idx.end(), blockable);
  int nblk = 0;
  while (nblk < static_cast<int>(batch->idx.size()) && blockable(batch->idx[nblk])) ++nblk;
  const int zstride = nblk > 0 ? std::max(steps, kTprsBlockDim) : steps;
  // offsets, then the locations and row mappings written straight into
  // page-locked staging by the host threads
  std::vector<int64_t> uoff, voff, roff;
  batch->nus.clear();
  int nu_max_blk = 0, nu_max = 0;
  int64_t vtotal = 0, utotal = 0, ltotal = 0;
  for (size_t c = 0; c < batch->idx.size(); ++c) {
    const TprsPrep& pr = batch->preps[batch->idx[c]];
    const bool blk = static_cast<int>(c) < nblk;
    uoff.push_back(ltotal);
    ltotal += static_cast<int64_t>(pr.u.size());
    batch->nus.push_back(pr.nu);
    voff.push_back(vtotal);
    vtotal += static_cast<int64_t>(pr.nu) * (blk ? kTprsBlockDim : steps);
    roff.push_back(utotal);
    utotal += static_cast<int64_t>(pr.nu) * kk;
    (blk ? nu_max_blk : nu_max) = std::max(blk ? nu_max_blk : nu_max, pr.nu);
  }
  double* hu = static_cast<double*>(stage_alloc(sizeof(double) * static_cast<size_t>(ltotal)));
  int* hmap = static_cast<int*>(stage_alloc(sizeof(int) * batch->idx.size() * static_cast<size_t>(n)));
  parallel_for(batch->idx.size(), [&](size_t c) {
    const TprsPrep& pr = batch->preps[batch->idx[c]];
    std::memcpy(hu + uoff[c], pr.u.data(), pr.u.size() * sizeof(double));
    std::memcpy(hmap + c * static_cast<size_t>(n), pr.mapping.data(), static_cast<size_t>(n) * sizeof(int));
  });
  const int cnt = static_cast<int>(batch->idx.size());
  const int nsingle = cnt - nblk;
  const int ctas = std::min(nsingle, ctas_per_sm * sms_);
  const int ctas_blk = std::min(nblk, 2 * sms_);  // two CTAs per SM (their shared memory)
  const size_t nab = static_cast<size_t>(2) * nsingle * steps;
  const size_t nvals = static_cast<size_t>(cnt) * kk;
  const size_t ns = static_cast<size_t>(cnt) * (kk - 1) * (kk - 1);
  const size_t ncs = static_cast<size_t>(cnt) * (kk - 1);
  // page-locked landing area: penalties, column sums of squares, status
  double* host = static_cast<double*>(stage_alloc(sizeof(double) * (ns + ncs + (static_cast<size_t>(cnt) + 1) / 2)));
  batch->S = host;
  batch->colsq = host + ns;
  batch->status = reinterpret_cast<int*>(host + ns + ncs);
  cuda_check(cudaMemcpyAsync(tb.u.ensure(static_cast<size_t>(ltotal)), hu, sizeof(double) * ltotal,
                             cudaMemcpyHostToDevice, st),
             "upload");
  cuda_check(cudaMemcpyAsync(tb.map.ensure(batch->idx.size() * static_cast<size_t>(n)), hmap,
                             sizeof(int) * batch->idx.size() * n, cudaMemcpyHostToDevice, st),
             "upload");
  stage_upload(tb.uoff, uoff, st);
  stage_upload(tb.voff, voff, st);
  stage_upload(tb.roff, roff, st);
  stage_upload(tb.nus, batch->nus, st);
  const int64_t ews_stride = tprs_ld(nu_max) * tprs_ld(nu_max);
  const int64_t ews_stride_blk = tprs_ld(nu_max_blk) * tprs_ld(nu_max_blk);
  double* dV = tb.V.ensure(static_cast<size_t>(vtotal));
  double* dab = tb.ab.ensure(std::max<size_t>(nab, 1));
  double* dblocks = tb.blocks.ensure(std::max<size_t>(static_cast<size_t>(nblk) * kTprsBlockSteps * 32, 1));
  double* ews = tb.ews.ensure(std::max(static_cast<size_t>(ctas) * ews_stride,
                                       static_cast<size_t>(ctas_blk) * ews_stride_blk));
  int* ddone = tb.done.ensure(cnt);
  double* dvals = tb.vals.ensure(nvals);
  double* dU = tb.U.ensure(static_cast<size_t>(utotal));
  int* dok = tb.ok.ensure(cnt);
  // a spare chunk from an earlier cache when one is large enough, else a new one
  const size_t xneed = static_cast<size_t>(cnt) * n * kk;
  std::unique_ptr<DevBuf<double>> chunk;
  for (size_t i = 0; i < smooth_spare_.size(); ++i)
    if (smooth_spare_[i]->capacity() >= xneed) {
      chunk = std::move(smooth_spare_[i]);
      smooth_spare_.erase(smooth_spare_.begin() + static_cast<std::ptrdiff_t>(i));
      break;
    }
  if (!chunk) chunk.reset(new DevBuf<double>());
  double* dX = chunk->ensure(xneed);
  smooth_store_.push_back(std::move(chunk));
  batch->X = dX;
  double* dS = tb.S.ensure(ns);
  double* dcs = tb.colsq.ensure(ncs);
  int* dst = tb.status.ensure(cnt);
  double* dzsel = tb.zsel.ensure(nvals * zstride);
  cuda_check(launch_tprs_block_lanczos(tb.u.get(), tb.uoff.get(), tb.nus.get(), nblk, nu_max_blk, tprs_eta0(dim),
                                       ews, ews_stride_blk, ctas_blk, dV, tb.voff.get(), dblocks, ddone, st),
             "thin-plate block Lanczos");
  cuda_check(launch_tprs_lanczos(tb.u.get(), tb.uoff.get() + nblk, tb.nus.get() + nblk, nsingle, nu_max, dim, steps,
                                 tprs_eta0(dim), ews, ews_stride, ctas, dV, tb.voff.get() + nblk, dab,
                                 dab + static_cast<size_t>(nsingle) * steps, ddone + nblk, st),
             "thin-plate Lanczos");
  cuda_check(launch_tprs_ritz_block_select(dblocks, ddone, nblk, kk, zstride,
                                           tb.ritzp.ensure(tprs_ritz_block_workspace(nblk)), dvals, dzsel, dok, st),
             "thin-plate Ritz pairs");
  cuda_check(launch_tprs_ritz_select(dab, dab + static_cast<size_t>(nsingle) * steps, ddone + nblk, nsingle, steps,
                                     kk, zstride, dvals + static_cast<size_t>(nblk) * kk,
                                     dzsel + static_cast<size_t>(nblk) * kk * zstride, dok + nblk, st),
             "thin-plate Ritz pairs");
  cuda_check(launch_tprs_ritz_vectors(dV, tb.voff.get(), tb.nus.get(), ddone, dok, dzsel, cnt, zstride, kk, dU,
                                      tb.roff.get(), st),
             "thin-plate Ritz vectors");
  cuda_check(launch_tprs_finish(dU, tb.roff.get(), dvals, dok, tb.u.get(), tb.uoff.get(),
                                tb.nus.get(), tb.map.get(), n, cnt, dim, dX, dS, dcs, dst, st),
             "thin-plate basis");
  cuda_check(cudaMemcpyAsync(batch->S, dS, ns * sizeof(double), cudaMemcpyDeviceToHost, st), "download");
  cuda_check(cudaMemcpyAsync(batch->colsq, dcs, ncs * sizeof(double), cudaMemcpyDeviceToHost, st), "download");
  cuda_check(cudaMemcpyAsync(batch->status, dst, static_cast<size_t>(cnt) * sizeof(int), cudaMemcpyDeviceToHost,
                             st),
             "download");
  d2h_bytes_ += static_cast<double>(ns + ncs) * sizeof(double) + static_cast<double>(cnt) * sizeof(int);
  cuda_check(cudaEventRecord(ev_[dim == 2 ? 6 : 7], st), "event");
}

void Engine::tprs_export(int a, int b, int* nu, int* path, int* ok, std::vector<double>* vals,
                         std::vector<double>* U) {
  if (a < 0 || b < 0 || a >= p_ || b >= p_ || a == b)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "a bivariate smooth needs two distinct columns of the data");
  release_graph();
  cuda_check(cudaStreamSynchronize(stream_), "set-up");
  stage_reset();
  TprsBatch batch;
  launch_tprs_batch({{std::min(a, b), std::max(a, b)}}, 2, &batch, stream_, tuning_.tprs_ctas_per_sm);
  *nu = batch.preps.empty() ? 0 : batch.preps[0].nu;
  *path = 0;
  *ok = 0;
  vals->clear();
  U->clear();
  if (batch.idx.empty()) {
    cuda_check(cudaStreamSynchronize(stream_), "thin-plate set-up");
    return;
  }
  const int n_u = batch.nus[0];
  *path = n_u >= kTprsBlockMinNu && tprs_ld(n_u) <= kTprsBlockMaxLd ? 2 : 1;
  TprsBuffers& tb = tprs_buf_[1];
  vals->assign(kTprsK, 0.0);
  U->assign(static_cast<size_t>(n_u) * kTprsK, 0.0);
  cuda_check(cudaMemcpyAsync(ok, tb.ok.get(), sizeof(int), cudaMemcpyDeviceToHost, stream_), "download");
  cuda_check(cudaMemcpyAsync(vals->data(), tb.vals.get(), sizeof(double) * kTprsK, cudaMemcpyDeviceToHost, stream_),
             "download");
  cuda_check(cudaMemcpyAsync(U->data(), tb.U.get(), sizeof(double) * U->size(), cudaMemcpyDeviceToHost, stream_),
             "download");
  cuda_check(cudaStreamSynchronize(stream_), "thin-plate set-up");
}

void Engine::finish_tprs_batch(TprsBatch* batch) {
  if (batch->idx.empty()) return;
  const int dim = batch->dim;
  cuda_check(cudaEventSynchronize(ev_[dim == 2 ? 6 : 7]), "thin-plate set-up");
  const int n = n_;
  const int kk = dim == 2 ? kTprsK : kTprsUniK;
  const int cols = kk - 1;
  std::vector<std::shared_ptr<Smooth>> made(batch->idx.size());
  // not converged or degenerate (status != 0): the host set-up builds that smooth
  parallel_for(batch->idx.size(), [&](size_t c) {
    if (batch->status[c] != 0) return;
    auto sm = std::make_shared<Smooth>();
    sm->n = n;
    sm->cols = cols;
    sm->rank = kk - (dim == 2 ? 3 : 2);  // the m = 2 thin plate's null space: 1, x (, y)
    sm->S.assign(batch->S + c * cols * cols, batch->S + (c + 1) * cols * cols);
    sm->colsq.assign(batch->colsq + c * cols, batch->colsq + (c + 1) * cols);
    if (dim == 1) sm->root = penalty_root(sm->S, cols, sm->rank);
    sm->dev_x = batch->X + c * static_cast<size_t>(n) * kk;
    made[c] = sm;
  });
  for (size_t c = 0; c < batch->idx.size(); ++c) {
    if (!made[c]) continue;
    const std::vector<int>& set = batch->sets[batch->idx[c]];
    if (dim == 2) cache_->put_bivariate(set, made[c]);
    else cache_->put_univariate(set[0], made[c]);
  }
}

// Designs of the sets selected by `pick`, built on host threads (the cache
// builds each conditioning set once).
template <class Pick>
void Engine::build_host_designs(Pick pick) {
  std::vector<size_t> todo;
  std::vector<const std::vector<int>*> keys;
  for (size_t i = 0; i < sets_.size(); ++i)
    if (!designs_[i] && pick(sets_[i])) {
      todo.push_back(i);
      keys.push_back(&sets_[i]);
    }
  if (todo.empty()) return;
  std::vector<std::shared_ptr<const Design>> found = cache_->find_designs(keys);
  std::vector<std::shared_ptr<const Design>> built(todo.size());
  std::string err;
  std::mutex err_mu;
  parallel_for(todo.size(), [&](size_t c) {
    if (found[c]) return;
    try {
      built[c] = cache_->build(sets_[todo[c]]);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (err.empty()) err = e.what();
    }
  });
  if (!err.empty()) throw Error(FKPC_STATUS_RANK, "design set-up failed: " + err);
  cache_->put_designs(keys, built);
  for (size_t c = 0; c < todo.size(); ++c) designs_[todo[c]] = found[c] ? found[c] : built[c];
}

// The univariate smooths of the batch's variables, each built once (several
// additive designs share a variable; building them design by design would
// let threads race to build the same smooth).
std::vector<std::vector<int>> Engine::univariate_columns() {
  std::vector<char> need(p_, 0);
  for (const auto& S : sets_)
    if (S.size() != 2)
      for (int v : S)
        if (v >= 0 && v < p_) need[v] = 1;
  std::vector<std::vector<int>> cols;
  for (int v = 0; v < p_; ++v)
    if (need[v] && !cache_->has_univariate(v)) cols.push_back({v});
  return cols;
}

void Engine::build_univariate_smooths() {
  std::vector<int> cols;
  for (const auto& c : univariate_columns()) cols.push_back(c[0]);
  std::string err;
  std::mutex err_mu;
  parallel_for(cols.size(), [&](size_t i) {
    try {
      cache_->univariate(cols[i]);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (err.empty()) err = e.what();
    }
  });
  if (!err.empty()) throw Error(FKPC_STATUS_RANK, "design set-up failed: " + err);
}

void Engine::build_designs() {
  designs_.assign(sets_.size(), nullptr);
  std::vector<std::vector<int>> bivariate;
  for (const auto& S : sets_)
    if (S.size() == 2 && !cache_->has_design(S)) bivariate.push_back(S);
  TprsBatch ubatch, batch;
  launch_tprs_batch(univariate_columns(), 1, &ubatch, stream_, tuning_.tprs_ctas_per_sm);
  if (bivariate.size() >= kDeviceTprsMin) launch_tprs_batch(bivariate, 2, &batch, stream_, tuning_.tprs_ctas_per_sm);
  // the other designs need no bivariate basis: build them while the device works
  finish_tprs_batch(&ubatch);
  build_univariate_smooths();  // those the device could not take
  build_host_designs([](const std::vector<int>& S) { return S.size() != 2; });
  finish_tprs_batch(&batch);
  build_host_designs([](const std::vector<int>& S) { return S.size() == 2; });
}

void Engine::pack_and_upload(const fkpc_options& opt, RStream* rstream, bool defer) {
  const int n = n_;
  // Pass 1: descriptors and arena offsets (no copies).  The arena has a
  // host-filled range [0, total) and, behind it, a device-filled range for the
  // geometry the device builds (offsets relative to the range while counting,
  // made absolute below).  The host range also holds the table of smooth
  // bases and penalties the geometry kernels read.
  // A design still null is a bivariate one whose basis the device is still
  // building: it gets its arena slots now (every bivariate design has
  // q = kTprsK and one penalty of rank kTprsK - 3) and the rest in pack_late.
  std::vector<DesignDev>& ddesc = ddesc_;
  ddesc.assign(designs_.size(), DesignDev());
  pending_.clear();
  std::vector<size_t> geom_designs, single_designs;
  size_t total = 0, dev_total = 0;
  struct SmoothSlot {
    const Smooth* smooth;
    int64_t x, pen;  // arena offsets of X (n x cols) and S (cols x cols, or -1)
  };
  std::vector<SmoothSlot> smooth_slots;
  std::map<const Smooth*, size_t> smooth_index;
  auto smooth_slot = [&](const Smooth* sm, bool with_penalty) -> SmoothSlot& {
    auto it = smooth_index.find(sm);
    if (it == smooth_index.end()) {
      it = smooth_index.emplace(sm, smooth_slots.size()).first;
      smooth_slots.push_back({sm, sm->dev_x ? -1 : static_cast<int64_t>(total), -1});
      total += sm->X.size();  // empty for a basis already on the device
    }
    SmoothSlot& sl = smooth_slots[it->second];
    if (with_penalty && sl.pen < 0) {
      sl.pen = static_cast<int64_t>(total);
      total += sm->S.size();
    }
    return sl;
  };
  // designs with more than kCtaPenalties blocks: their full descriptors,
  // copied into the host range of the arena at ``ext``
  std::vector<std::pair<size_t, WideDesign>> wide_desc;
  // penalty roots in the host range, one per distinct root vector
  std::map<const std::vector<double>*, int64_t> root_slot;
  std::vector<std::pair<const std::vector<double>*, int64_t>> root_copies;
  for (size_t d = 0; d < designs_.size(); ++d) {
    DesignDev& dd = ddesc[d];
    std::memset(&dd, 0, sizeof(dd));
    dd.ext = -1;
    if (!designs_[d]) {
      if (sets_[d].size() != 2) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "design set-up incomplete");
      dd.kind = 1;
      dd.q = kTprsK;
      dd.m = 1;
      dd.basis = static_cast<int64_t>(dev_total);
      dev_total += static_cast<size_t>(n) * kTprsK;
      dd.spec = static_cast<int64_t>(dev_total);
      dev_total += kTprsK;
      dd.off[0] = 1;
      dd.dim[0] = kTprsK - 1;
      dd.rank[0] = kTprsK - 3;
      dd.rsum = kTprsK - 3;
      pending_.push_back(d);
      continue;
    }
    const Design& des = *designs_[d];
    dd.q = des.q;
    dd.m = des.m;
    if (des.m == 1) {
      if (des.q > kMaxSingleQ) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "single-penalty design too wide");
      dd.kind = 1;
      size_t& at = des.device_geometry ? dev_total : total;
      dd.basis = static_cast<int64_t>(at);
      at += static_cast<size_t>(n) * des.q;
      dd.spec = static_cast<int64_t>(at);
      at += static_cast<size_t>(des.q);
      if (des.device_geometry) {
        single_designs.push_back(d);
        smooth_slot(des.parts[0].get(), true);
      }
      dd.log_sp0[0] = des.initial_log_sp[0];
      dd.off[0] = des.offsets[0];
      dd.dim[0] = des.dims[0];
      dd.rank[0] = des.ranks[0];
      dd.rsum = des.ranks[0];
    } else {
      dd.kind = 2;
      const bool dev = des.device_geometry;
      size_t& at = dev ? dev_total : total;
      dd.basis = static_cast<int64_t>(at);
      at += static_cast<size_t>(n) * des.q;
      dd.rmat = static_cast<int64_t>(at);
      at += static_cast<size_t>(des.q) * des.q;
      // the roots: one copy per univariate smooth, shared by every design
      // that contains the variable (absolute offsets, roots = 0); a block
      // whose root is not its smooth's own gets a copy of its own
      dd.roots = 0;
      if (des.m > kMaxPenalties)
        throw Error(FKPC_STATUS_INVALID_ARGUMENT, "additive design exceeds the kernel capacity (q <= 560, |S| <= 62)");
      WideDesign wd;
      std::memset(&wd, 0, sizeof(wd));
      int rows = 0;
      for (int j = 0; j < des.m; ++j) {
        const Smooth* part = j < static_cast<int>(des.parts.size()) ? des.parts[j].get() : nullptr;
        const std::vector<double>* src = &des.roots[j];
        if (part && part->root == des.roots[j]) src = &part->root;
        auto it = root_slot.find(src);
        if (it == root_slot.end()) {
          it = root_slot.emplace(src, static_cast<int64_t>(total)).first;
          root_copies.push_back({src, static_cast<int64_t>(total)});
          total += src->size();
        }
        if (it->second > INT32_MAX) throw Error(FKPC_STATUS_ALLOCATION, "penalty roots beyond the arena's int32 offsets");
        wd.off[j] = des.offsets[j];
        wd.dim[j] = des.dims[j];
        wd.rank[j] = des.ranks[j];
        wd.rowoff[j] = rows;
        wd.rootoff[j] = static_cast<int>(it->second);
        wd.log_sp0[j] = des.initial_log_sp[j];
        rows += des.ranks[j];
      }
      for (int j = 0; j < des.m && j < kCtaPenalties; ++j) {
        dd.off[j] = wd.off[j];
        dd.dim[j] = wd.dim[j];
        dd.rank[j] = wd.rank[j];
        dd.rowoff[j] = wd.rowoff[j];
        dd.rootoff[j] = wd.rootoff[j];
        dd.log_sp0[j] = wd.log_sp0[j];
      }
      dd.rsum = rows;
      if (des.m > kCtaPenalties) {
        dd.ext = static_cast<int64_t>(total);
        total += sizeof(WideDesign) / sizeof(double);
        wide_desc.emplace_back(d, wd);
      }
      if (des.q > kWideQ || rows > kWideR)
        throw Error(FKPC_STATUS_INVALID_ARGUMENT, "additive design exceeds the kernel capacity (q <= 560, |S| <= 62)");
      if (des.q >= n_)
        throw Error(FKPC_STATUS_INVALID_ARGUMENT, "additive design has at least as many coefficients as observations (q = " +
                                                      std::to_string(des.q) + ", n = " + std::to_string(n_) + ")");
      dd.rpack = -1;
      if (des.q <= kWarpQ) {
        size_t& pat = dev ? dev_total : total;
        pat += pat % 2;  // 16-byte aligned: copied with 16-byte cp.async
        dd.rpack = static_cast<int64_t>(pat);
        pat += kWarpTri;
      }
      if (dev) {
        geom_designs.push_back(d);
        for (const auto& sm : des.parts) smooth_slot(sm.get(), false);
      }
    }
  }
  const size_t dev_base = total + total % 2;  // keeps the device range's rpack offsets 16-byte aligned
  for (size_t d : geom_designs) {
    DesignDev& dd = ddesc[d];
    dd.basis += static_cast<int64_t>(dev_base);
    dd.rmat += static_cast<int64_t>(dev_base);
    if (dd.rpack >= 0) dd.rpack += static_cast<int64_t>(dev_base);
  }
  for (size_t d : single_designs) {
    ddesc[d].basis += static_cast<int64_t>(dev_base);
    ddesc[d].spec += static_cast<int64_t>(dev_base);
  }
  for (size_t d : pending_) {
    ddesc[d].basis += static_cast<int64_t>(dev_base);
    ddesc[d].spec += static_cast<int64_t>(dev_base);
  }
  for (auto& [d, wd] : wide_desc) {  // the header with its final arena offsets
    const DesignDev& dd = ddesc[d];
    wd.kind = dd.kind;
    wd.q = dd.q;
    wd.m = dd.m;
    wd.rsum = dd.rsum;
    wd.basis = dd.basis;
    wd.rmat = dd.rmat;
    wd.spec = dd.spec;
    wd.roots = dd.roots;
    wd.rpack = dd.rpack;
    wd.ext = dd.ext;
  }
  // Pass 2: every design copies its host-built part into the pinned staging
  // buffer (threads over designs), then one DMA to the device arena.
  double* host = pinned_arena(total);
  for (const auto& [d, wd] : wide_desc) std::memcpy(host + ddesc[d].ext, &wd, sizeof(WideDesign));
  for (const auto& [src, at] : root_copies) std::memcpy(host + at, src->data(), src->size() * sizeof(double));
  {
    std::atomic<size_t> next(0);
    auto work = [&]() {
      for (;;) {
        const size_t item = next.fetch_add(1);
        if (item >= designs_.size() + smooth_slots.size()) return;
        if (item >= designs_.size()) {
          const SmoothSlot& sl = smooth_slots[item - designs_.size()];
          if (sl.x >= 0) std::memcpy(host + sl.x, sl.smooth->X.data(), sl.smooth->X.size() * sizeof(double));
          if (sl.pen >= 0) std::memcpy(host + sl.pen, sl.smooth->S.data(), sl.smooth->S.size() * sizeof(double));
          continue;
        }
        const size_t d = item;
        if (!designs_[d]) continue;  // pending: nothing on the host yet
        const Design& des = *designs_[d];
        const DesignDev& dd = ddesc[d];
        if (dd.kind == 1) {
          if (des.device_geometry) continue;
          std::memcpy(host + dd.basis, des.QW.data(), des.QW.size() * sizeof(double));
          std::memcpy(host + dd.spec, des.spec.data(), des.spec.size() * sizeof(double));
        } else {
          if (des.device_geometry) continue;  // its roots are the shared copies above
          std::memcpy(host + dd.basis, des.Q.data(), des.Q.size() * sizeof(double));
          std::memcpy(host + dd.rmat, des.R.data(), des.R.size() * sizeof(double));
          if (dd.rpack >= 0) {
            double* rp = host + dd.rpack;
            std::fill(rp, rp + kWarpTri, 0.0);
            for (int t = 0; t < des.q; ++t)
              for (int c = t; c < des.q; ++c) rp[packed_row(t, c)] = des.R[t + static_cast<size_t>(des.q) * c];
          }
        }
      }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t workers =
        std::min<size_t>(std::min<size_t>(hw, 16), std::max<size_t>(1, (designs_.size() + smooth_slots.size()) / 64));
    if (workers <= 1) {
      work();
    } else {
      std::vector<std::thread> pool;
      for (size_t w = 0; w < workers; ++w) pool.emplace_back(work);
      for (auto& th : pool) th.join();
    }
  }
  // Device geometry jobs; the smooth bases and penalties sit in the host range
  // (a bivariate basis built on the device stays in the smooth store).
  double* arena = d_arena_.ensure(dev_base + dev_total);
  std::vector<GeomJob> gjobs;
  std::vector<WideGeomJob> wgjobs;
  std::vector<SingleGeomJob> sjobs(single_designs.size());
  int geom_max_q = 1;
  for (size_t g = 0; g < single_designs.size(); ++g) {
    const Design& des = *designs_[single_designs[g]];
    const DesignDev& dd = ddesc[single_designs[g]];
    const SmoothSlot& sl = smooth_slots[smooth_index.at(des.parts[0].get())];
    SingleGeomJob& job = sjobs[g];
    std::memset(&job, 0, sizeof(job));
    job.basis = dd.basis;
    job.spec = dd.spec;
    job.src = sl.smooth->dev_x ? sl.smooth->dev_x : arena + sl.x;
    job.pen = arena + sl.pen;
    job.q = des.q;
    job.rank = des.ranks[0];
  }
  int wide_max_q = 1;
  auto fill_geom = [&](auto& job, const Design& des, const DesignDev& dd) {
    std::memset(&job, 0, sizeof(job));
    job.basis = dd.basis;
    job.rmat = dd.rmat;
    job.rpack = dd.rpack;
    job.q = des.q;
    job.m = des.m;
    for (int j = 0; j < des.m; ++j) {
      const Smooth* sm = des.parts[j].get();
      job.src[j] = sm->dev_x ? sm->dev_x : arena + smooth_slots[smooth_index.at(sm)].x;
      job.off[j] = des.offsets[j];
      job.dim[j] = des.dims[j];
    }
  };
  for (size_t g = 0; g < geom_designs.size(); ++g) {
    const Design& des = *designs_[geom_designs[g]];
    const DesignDev& dd = ddesc[geom_designs[g]];
    if (des.m > kCtaPenalties) {
      wgjobs.emplace_back();
      fill_geom(wgjobs.back(), des, dd);
      wide_max_q = std::max(wide_max_q, des.q);
    } else {
      gjobs.emplace_back();
      fill_geom(gjobs.back(), des, dd);
      geom_max_q = std::max(geom_max_q, des.q);
    }
  }
  // Widest designs first: the geometry kernel's CTAs take jobs in a fixed
  // stride and a QR costs about n q^2, so the last jobs of every CTA are the
  // short ones.  Each job writes only its own arena ranges; status is checked
  // as a whole.
  std::stable_sort(gjobs.begin(), gjobs.end(), [](const GeomJob& a, const GeomJob& b) { return a.q > b.q; });
  single_jobs_.clear();
  multi_jobs_.clear();
  multi_small_.clear();
  multi_large_.clear();
  multi_huge_.clear();
  multi_wide_.clear();
  direct_cols_.clear();
  direct_slots_.clear();
  plain_single_off_.clear();
  plain_small_off_.clear();
  plain_large_off_.clear();
  plain_huge_off_.clear();
  plain_wide_off_.clear();
  plain_direct_off_.clear();
  for (size_t c = 0; c < comps_.size(); ++c) {
    if (opt.mode == FKPC_MODE_PLAIN && c % 2 == 0) {
      plain_single_off_.push_back(static_cast<int>(single_jobs_.size()));
      plain_small_off_.push_back(static_cast<int>(multi_small_.size()));
      plain_large_off_.push_back(static_cast<int>(multi_large_.size()));
      plain_huge_off_.push_back(static_cast<int>(multi_huge_.size()));
      plain_wide_off_.push_back(static_cast<int>(multi_wide_.size()));
      plain_direct_off_.push_back(static_cast<int>(direct_cols_.size()));
    }
    const Component& cp = comps_[c];
    if (cp.design < 0) {
      direct_cols_.push_back(cp.target);
      direct_slots_.push_back(static_cast<int>(c));
      continue;
    }
    FitJob job{cp.design, cp.target, static_cast<int>(c), 0};
    const DesignDev& dd = ddesc[cp.design];
    if (dd.kind == 1) {
      single_jobs_.push_back(job);
    } else {
      const int idx = static_cast<int>(multi_jobs_.size());
      multi_jobs_.push_back(job);
      if (dd.q <= kWarpQ && dd.rsum <= kWarpR && dd.m <= kWarpM) multi_small_.push_back(idx);
      else if (dd.q <= 76 && dd.rsum <= 64 && dd.m <= kCtaPenalties) multi_large_.push_back(idx);
      else if (dd.q <= 112 && dd.rsum <= 96 && dd.m <= kCtaPenalties) multi_huge_.push_back(idx);
      else if (dd.ext >= 0) multi_wide_.push_back(idx);
      else throw Error(FKPC_STATUS_INVALID_ARGUMENT, "additive design fits no fit class");
    }
  }
  if (opt.mode != FKPC_MODE_PLAIN) {
    // Longest fits first: the warp fit kernel's CTAs start in index order, so
    // the widest designs (an evaluation costs about q^2) leave the last wave
    // to the short ones.  Results are written by job index; order is free.
    std::stable_sort(multi_small_.begin(), multi_small_.end(), [&](int a, int b) {
      return ddesc[multi_jobs_[a].design].q > ddesc[multi_jobs_[b].design].q;
    });
  }
  if (opt.mode == FKPC_MODE_PLAIN) {
    plain_single_off_.push_back(static_cast<int>(single_jobs_.size()));
    plain_small_off_.push_back(static_cast<int>(multi_small_.size()));
    plain_large_off_.push_back(static_cast<int>(multi_large_.size()));
    plain_huge_off_.push_back(static_cast<int>(multi_huge_.size()));
    plain_wide_off_.push_back(static_cast<int>(multi_wide_.size()));
    plain_direct_off_.push_back(static_cast<int>(direct_cols_.size()));
  }
  const size_t ncomp = comps_.size();
  const size_t npairs = pairs_.size();
  auto t0 = std::chrono::steady_clock::now();
  h2d_bytes_ = static_cast<double>(host_data_.size() * sizeof(double));
  if (total > 0)
    cuda_check(cudaMemcpyAsync(arena, host, total * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload arena");
  h2d_bytes_ += static_cast<double>(total * sizeof(double));
  int* gstatus_dev = d_geom_status_.ensure(gjobs.size() + wgjobs.size() + sjobs.size() + pending_.size());
  geom_status_used_ = gjobs.size() + wgjobs.size() + sjobs.size();
  geom_status_checked_ = 0;
  if (!gjobs.empty()) {
    h2d_bytes_ += stage_upload(d_geom_jobs_, gjobs);
    cuda_check(launch_additive_geometry(n, d_geom_jobs_.get(), static_cast<int>(gjobs.size()), geom_max_q, arena,
                                        gstatus_dev, stream_),
               "additive geometry");
  }
  if (!wgjobs.empty()) {
    h2d_bytes_ += stage_upload(d_wide_geom_jobs_, wgjobs);
    cuda_check(launch_additive_geometry(n, d_wide_geom_jobs_.get(), static_cast<int>(wgjobs.size()), wide_max_q, arena,
                                        gstatus_dev + gjobs.size(), stream_),
               "additive geometry");
  }
  if (!sjobs.empty()) {
    h2d_bytes_ += stage_upload(d_single_geom_jobs_, sjobs);
    cuda_check(launch_single_geometry(n, d_single_geom_jobs_.get(), static_cast<int>(sjobs.size()), arena,
                                      gstatus_dev + gjobs.size() + wgjobs.size(), stream_),
               "single-penalty geometry");
  }
  h2d_bytes_ += stage_upload(d_designs_, ddesc);
  h2d_bytes_ += stage_upload(d_single_jobs_, single_jobs_);
  h2d_bytes_ += stage_upload(d_multi_jobs_, multi_jobs_);
  h2d_bytes_ += stage_upload(d_multi_small_, multi_small_);
  h2d_bytes_ += stage_upload(d_multi_large_, multi_large_);
  h2d_bytes_ += stage_upload(d_multi_huge_, multi_huge_);
  h2d_bytes_ += stage_upload(d_multi_wide_, multi_wide_);
  if (!multi_small_.empty()) {
    d_fit_states_.ensure(multi_jobs_.size());
    d_defer_list_.ensure(multi_small_.size());
    d_defer_count_.ensure(1);
  }
  if (!multi_huge_.empty() || !multi_wide_.empty())
    d_fit_ws_.ensure(std::max(multi_workspace_doubles(2, static_cast<int>(multi_huge_.size())),
                              multi_workspace_doubles(3, static_cast<int>(multi_wide_.size()))));
  if (!multi_wide_.empty()) d_wide_log_sp_.ensure(multi_wide_.size() * static_cast<size_t>(kMaxPenalties));
  h2d_bytes_ += stage_upload(d_direct_cols_, direct_cols_);
  h2d_bytes_ += stage_upload(d_direct_slots_, direct_slots_);
  h2d_bytes_ += stage_upload(d_pairs_, pairs_);
  std::vector<int> ident(ncomp);
  for (size_t c = 0; c < ncomp; ++c) ident[c] = static_cast<int>(c);
  h2d_bytes_ += stage_upload(d_comp_cols_, ident);
  collected_ = false;
  d_single_res_.ensure(single_jobs_.size());
  d_multi_res_.ensure(multi_jobs_.size());
  d_resid_.ensure(static_cast<size_t>(n) * ncomp);
  d_records_.ensure(npairs);
  d_late_col_.ensure(ncomp);
  d_part_.ensure(4 + 2 * ncomp + 2 * npairs);
  d_guard_mark_.ensure(2);
  late_designs_ = false;  // a new batch: the descriptor array of the side stream is stale
  if (stats_enabled_) {
    const int method = opt.ci_method;
    if (method == FKPC_DCC_GAMMA || method == FKPC_DCC_PERM) {
      d_centre_.ensure(static_cast<size_t>(n) * ncomp);
      d_dcov_.ensure(ncomp);
    }
    if (method == FKPC_HSIC_GAMMA || method == FKPC_HSIC_PERM) {
      d_factors_.ensure(static_cast<size_t>(n) * opt.num_col * ncomp);
      d_hsic_.ensure(ncomp);
    }
    if (method == FKPC_DCC_GAMMA) {
      const size_t bytes_per_slot = static_cast<size_t>(n) * opt.num_col * sizeof(double);
      const size_t budget = static_cast<size_t>(8) << 30;
      guard_cap_ = static_cast<int>(std::min<size_t>(ncomp, std::max<size_t>(1, budget / bytes_per_slot)));
      d_guard_.ensure(2 + npairs + ncomp + guard_cap_);
      d_lr_vals_.ensure(static_cast<size_t>(guard_cap_) * opt.num_col);
      d_lr_vecs_.ensure(static_cast<size_t>(guard_cap_) * opt.num_col * n);
      d_lr_status_.ensure(2 * static_cast<size_t>(guard_cap_));
      d_legacy_ws_.ensure(legacy_eigen_workspace_doubles(n, legacy_ctas()));
      lr_ws_ctas_ = legacy_ctas();
    }
    if (method == FKPC_DCC_PERM || method == FKPC_HSIC_PERM) {
      if (!rstream) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation methods require a seeded stream");
      const int R = opt.permutation_replicates;
      std::vector<int> perms(npairs * static_cast<size_t>(R) * n);
      // the stream's draws test after test (sequential: one seeded stream),
      // then every test's table from its draws on the host threads
      for (size_t t = 0; t < npairs; ++t) {
        int* dst = perms.data() + t * static_cast<size_t>(R) * n;
        if (method == FKPC_DCC_PERM) rstream->dcc_swaps(n, R, dst);
        else rstream->hsic_draws(n, R, dst);
        if (stream_snapshots_) stream_snapshots_->push_back(*rstream);
      }
      parallel_for(npairs, [&](size_t t) {
        thread_local std::vector<int> scratch;
        int* dst = perms.data() + t * static_cast<size_t>(R) * n;
        if (method == FKPC_DCC_PERM) RStream::dcc_assemble(n, R, dst, &scratch);
        else RStream::hsic_assemble(n, R, dst, &scratch);
      });
      h2d_bytes_ += upload(d_perms_, perms, stream_);
    }
  }
  if (!defer) {
    cuda_check(cudaStreamSynchronize(stream_), "prepare upload");
    check_geometry();
  }
  upload_ms_ = ms_since(t0);
}

void Engine::check_geometry() {
  if (geom_status_used_ <= geom_status_checked_) return;
  std::vector<int> gstatus(geom_status_used_);
  cuda_check(cudaMemcpy(gstatus.data(), d_geom_status_.get(), gstatus.size() * sizeof(int), cudaMemcpyDeviceToHost),
             "download");
  geom_status_checked_ = geom_status_used_;
  for (int st : gstatus) {
    if (st == 1) throw Error(FKPC_STATUS_RANK, "design set-up failed: design matrix is rank deficient");
    if (st != 0) throw Error(FKPC_STATUS_NUMERIC, "design set-up failed: penalty eigen-decomposition did not converge");
  }
}

void Engine::pack_late(cudaStream_t st) {
  if (pending_.empty()) return;
  const bool side = st == side_;
  // the side stream reads the arena and the smooth store the main stream
  // filled before the fits were queued
  if (side) cuda_check(cudaStreamWaitEvent(side_, ev_[0], 0), "stream wait");
  const int n = n_;
  std::vector<double> late;  // penalties, and the bases a host fallback built
  std::vector<int64_t> xoff(pending_.size(), -1), poff(pending_.size(), -1);
  for (size_t g = 0; g < pending_.size(); ++g) {
    const size_t d = pending_[g];
    const Design& des = *designs_[d];
    if (des.m != 1 || des.q != kTprsK || !des.device_geometry || des.parts.empty())
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "bivariate design of an unexpected shape");
    DesignDev& dd = ddesc_[d];
    dd.log_sp0[0] = des.initial_log_sp[0];
    dd.off[0] = des.offsets[0];
    dd.dim[0] = des.dims[0];
    dd.rank[0] = des.ranks[0];
    dd.rsum = des.ranks[0];
    const Smooth& sm = *des.parts[0];
    if (!sm.dev_x) {
      xoff[g] = static_cast<int64_t>(late.size());
      late.insert(late.end(), sm.X.begin(), sm.X.end());
    }
    poff[g] = static_cast<int64_t>(late.size());
    late.insert(late.end(), sm.S.begin(), sm.S.end());
  }
  h2d_bytes_ += stage_upload(d_late_table_, late, st);
  const double* table = d_late_table_.get();
  std::vector<SingleGeomJob> jobs(pending_.size());
  for (size_t g = 0; g < pending_.size(); ++g) {
    const size_t d = pending_[g];
    const Design& des = *designs_[d];
    SingleGeomJob& job = jobs[g];
    std::memset(&job, 0, sizeof(job));
    job.basis = ddesc_[d].basis;
    job.spec = ddesc_[d].spec;
    job.src = des.parts[0]->dev_x ? des.parts[0]->dev_x : table + xoff[g];
    job.pen = table + poff[g];
    job.q = des.q;
    job.rank = des.ranks[0];
  }
  h2d_bytes_ += stage_upload(d_late_geom_jobs_, jobs, st);
  // the descriptor array again, now complete.  On the main stream it is
  // queued behind the multi-penalty fits, which read the additive
  // descriptors; beside them, on the side stream, it goes to a buffer of its
  // own, which the single-penalty fits read.
  if (side) {
    h2d_bytes_ += stage_upload(d_designs_late_, ddesc_, st);
    late_designs_ = true;
  } else {
    h2d_bytes_ += stage_upload(d_designs_, ddesc_, st);
  }
  cuda_check(launch_single_geometry(n, d_late_geom_jobs_.get(), static_cast<int>(jobs.size()), d_arena_.get(),
                                    d_geom_status_.get() + geom_status_used_, st),
             "single-penalty geometry");
  geom_status_used_ += jobs.size();
  pending_.clear();
}

void Engine::prepare(const std::vector<Test>& tests, const fkpc_options& opt, RStream* rstream) {
  if (n_ == 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "no data loaded");
  graph_timed_ = false;
  call_timed_ = false;
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaStreamSynchronize(stream_), "prepare");
  stage_reset();
  d2h_bytes_ = 0.0;
  opt_ = opt;
  stats_enabled_ = true;
  late_designs_ = false;
  release_graph();
  auto t0 = std::chrono::steady_clock::now();
  plan_components(tests);
  designs_built_ = 0;
  for (const auto& S : sets_) designs_built_ += cache_->has_design(S) ? 0 : 1;
  smooths_built_ = static_cast<int>(univariate_columns().size());
  build_designs();
  setup_ms_ = ms_since(t0);
  pack_and_upload(opt, rstream);
}

void Engine::run_batch(const std::vector<Test>& tests, const fkpc_options& opt, RStream* rstream) {
  if (n_ == 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "no data loaded");
  graph_timed_ = false;
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaStreamSynchronize(stream_), "batch");
  stage_reset();
  d2h_bytes_ = 0.0;
  opt_ = opt;
  stats_enabled_ = true;
  late_designs_ = false;
  release_graph();
  try {
    auto t0 = std::chrono::steady_clock::now();
    cuda_check(cudaEventRecord(ev_call_, stream_), "event");
    call_timed_ = true;
    plan_components(tests);
    designs_built_ = 0;
    for (const auto& S : sets_) designs_built_ += cache_->has_design(S) ? 0 : 1;
    smooths_built_ = static_cast<int>(univariate_columns().size());
    plan_ms_ = ms_since(t0);
    designs_.assign(sets_.size(), nullptr);
    std::vector<std::vector<int>> bivariate;
    for (const auto& S : sets_)
      if (S.size() == 2 && !cache_->has_design(S)) bivariate.push_back(S);
    // The univariate thin-plate batch (one CTA per variable: a third of the
    // SMs at p = 50) on the side stream, beside the bivariate one on the main
    // stream; the host waits for it before it builds the additive descriptors,
    // so everything the main stream queues after that sees its bases.  The
    // bivariate kernels stay on the main stream ahead of the fits: they hold
    // every SM, so on a second stream they would delay the multi-penalty fits
    // rather than run beside them.
    TprsBatch ubatch, batch;
    auto tp = std::chrono::steady_clock::now();
    launch_tprs_batch(univariate_columns(), 1, &ubatch, side_, tuning_.tprs_ctas_per_sm);
    if (!bivariate.empty()) launch_tprs_batch(bivariate, 2, &batch, stream_, tuning_.tprs_ctas_per_sm);
    tprs_host_ms_ = ms_since(tp);
    auto tw = std::chrono::steady_clock::now();
    finish_tprs_batch(&ubatch);
    smooth_wait_ms_ = ms_since(tw);
    auto td = std::chrono::steady_clock::now();
    build_univariate_smooths();  // those the device could not take
    build_host_designs([this](const std::vector<int>& S) { return S.size() != 2 || cache_->has_design(S); });
    design_host_ms_ = ms_since(td);
    double host_ms = ms_since(t0);
    pack_and_upload(opt, rstream, true);  // queued behind the univariate thin-plate kernels
    double up_ms = upload_ms_;
    cuda_check(configure_fit_kernels(), "kernel attributes");
    cuda_check(configure_stat_kernels(n_), "kernel attributes");
    launches_ = 0;
    cuda_check(cudaEventRecord(ev_[0], stream_), "event");
    enqueue_multi();
    auto t1 = std::chrono::steady_clock::now();
    finish_tprs_batch(&batch);
    late_wait_ms_ = ms_since(t1);
    auto td2 = std::chrono::steady_clock::now();
    build_host_designs([](const std::vector<int>&) { return true; });
    design_host_ms_ += ms_since(td2);
    host_ms += ms_since(t1);
    auto t2 = std::chrono::steady_clock::now();
    pack_late(split_stats() ? side_ : stream_);
    up_ms += ms_since(t2);
    enqueue_rest();
    setup_ms_ = host_ms;
    upload_ms_ = up_ms;
  } catch (...) {
    cudaStreamSynchronize(side_);  // nothing queued may outlive the call's staging
    cudaStreamSynchronize(stream_);
    throw;
  }
}

void Engine::enqueue() {
  launches_ = 0;
  cuda_check(cudaEventRecord(ev_[0], stream_), "event");
  enqueue_multi();
  enqueue_rest();
}

void Engine::enqueue_multi() {
  const int n = n_;
  // the CTA classes first: once the one-warp kernel is done, every fit but
  // the ones it hands to the speculative continuation is final
  if (!multi_large_.empty()) {
    cuda_check(launch_fit_multi(1, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_large_.get(), static_cast<int>(multi_large_.size()), d_resid_.get(),
                                d_multi_res_.get(), stream_, opt_.selection),
               "fit multi");
    ++launches_;
  }
  if (!multi_huge_.empty()) {
    cuda_check(launch_fit_multi(2, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_huge_.get(), static_cast<int>(multi_huge_.size()), d_resid_.get(),
                                d_multi_res_.get(), stream_, opt_.selection, d_fit_ws_.get()),
               "fit multi");
    ++launches_;
  }
  if (!multi_wide_.empty()) {  // after the q <= 112 class: the two share the workspace
    cuda_check(launch_fit_multi(3, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_wide_.get(), static_cast<int>(multi_wide_.size()), d_resid_.get(),
                                d_multi_res_.get(), stream_, opt_.selection, d_fit_ws_.get(), nullptr, nullptr,
                                nullptr, nullptr, 0, d_wide_log_sp_.get()),
               "fit multi");
    ++launches_;
  }
  const bool split = split_stats();
  if (!multi_small_.empty()) {
    cuda_check(launch_fit_multi(0, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_small_.get(), static_cast<int>(multi_small_.size()), d_resid_.get(),
                                d_multi_res_.get(), stream_, opt_.selection, nullptr, d_fit_states_.get(),
                                d_defer_list_.get(), d_defer_count_.get(), split ? ev_warp_ : nullptr,
                                tuning_.defer_evaluations),
               "fit multi");
    launches_ += opt_.selection == FKPC_SELECT_MAGIC ? 2 : 1;  // with the speculative continuation
  } else if (split) {
    cuda_check(cudaEventRecord(ev_warp_, stream_), "event");
  }
}

bool Engine::split_stats() const {
  return tuning_.split_statistics && stats_enabled_ && opt_.mode != FKPC_MODE_PLAIN && !pairs_.empty() &&
         (opt_.ci_method == FKPC_DCC_GAMMA || opt_.ci_method == FKPC_HSIC_GAMMA);
}

void Engine::enqueue_rest() {
  const int n = n_;
  const bool split = split_stats();
  // direct columns and single-penalty fits: on the side stream when the
  // statistics split, where they run beside the multi-penalty fits
  cudaStream_t fs = split ? side_ : stream_;
  if (split) cuda_check(cudaStreamWaitEvent(side_, ev_[0], 0), "stream wait");
  if (!direct_cols_.empty()) {
    dim3 grid((n + 255) / 256, static_cast<unsigned>(direct_cols_.size()));
    gather_columns_kernel<<<grid, 256, 0, fs>>>(d_data_.get(), n, d_direct_cols_.get(), d_direct_slots_.get(),
                                                 static_cast<int>(direct_cols_.size()), d_resid_.get());
    cuda_check(cudaGetLastError(), "gather columns");
    ++launches_;
  }
  if (!single_jobs_.empty()) {
    const DesignDev* designs = late_designs_ ? d_designs_late_.get() : d_designs_.get();
    cuda_check(launch_fit_single(designs, d_arena_.get(), d_data_.get(), n, d_single_jobs_.get(),
                                 static_cast<int>(single_jobs_.size()), d_resid_.get(), d_single_res_.get(), fs),
               "fit single");
    ++launches_;
  }
  if (!split) {
    cuda_check(cudaEventRecord(ev_[1], stream_), "event");
    enqueue_stats_serial();
    cuda_check(cudaEventRecord(ev_[3], stream_), "event");
    return;
  }
  const int ncomp = static_cast<int>(comps_.size());
  const int npairs = static_cast<int>(pairs_.size());
  const bool dcc = opt_.ci_method == FKPC_DCC_GAMMA;
  int* part = d_part_.get();
  const WorkList early_c{part + 4, part + 0}, late_c{part + 4 + ncomp, part + 1};
  const WorkList early_p{part + 4 + 2 * ncomp, part + 2}, late_p{part + 4 + 2 * ncomp + npairs, part + 3};
  int* guard = d_guard_.get();
  int* mark = d_guard_mark_.get();
  const int* glist = guard + 2;
  const int* comp_slot = glist + npairs;
  const int* slot_comps = comp_slot + ncomp;
  const int lr_ctas = lowrank_launch_ctas();
  // side stream, once the one-warp kernel is done: the early statistics
  cuda_check(cudaStreamWaitEvent(side_, ev_warp_, 0), "stream wait");
  const bool deferring = !multi_small_.empty() && opt_.selection == FKPC_SELECT_MAGIC && tuning_.defer_evaluations > 0;
  cuda_check(launch_stat_partition(deferring ? d_defer_list_.get() : nullptr,
                                   deferring ? d_defer_count_.get() : nullptr, d_multi_jobs_.get(), ncomp,
                                   d_pairs_.get(), npairs, d_late_col_.get(), part, side_),
             "partition");
  ++launches_;
  // the main stream reads the late lists the partition writes
  cuda_check(cudaEventRecord(ev_part_, side_), "event");
  if (dcc) {
    cuda_check(launch_dcov_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, d_centre_.get(), d_dcov_.get(),
                                      side_, early_c),
               "dcov components");
    cuda_check(launch_dcov_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_dcov_.get(),
                                 d_pairs_.get(), npairs, d_records_.get(), side_, early_p),
               "dcov pairs");
    cuda_check(launch_guard_select(d_records_.get(), d_pairs_.get(), npairs, ncomp, guard_cap_, kGuardLower,
                                   kGuardUpper, guard, side_, early_p),
               "guard select");
    cuda_check(launch_legacy_eigen(d_resid_.get(), n, d_comp_cols_.get(), guard, slot_comps, guard_cap_, lr_ctas,
                                   opt_.num_col, d_legacy_ws_.get(), d_lr_vals_.get(), d_lr_vecs_.get(),
                                   d_lr_status_.get(), side_),
               "legacy eigen");
    cuda_check(launch_legacy_pairs(n, opt_.num_col, d_lr_vals_.get(), d_lr_vecs_.get(), d_dcov_.get(), guard, glist,
                                   comp_slot, d_pairs_.get(), npairs, d_records_.get(), side_),
               "legacy pairs");
    launches_ += 5;
  } else {
    cuda_check(launch_hsic_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, opt_.num_col, opt_.hsic_sig,
                                      d_factors_.get(), d_hsic_.get(), side_, early_c),
               "hsic components");
    cuda_check(launch_hsic_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), d_pairs_.get(), npairs,
                                 d_records_.get(), side_, early_p),
               "hsic pairs");
    launches_ += 2;
  }
  cuda_check(cudaEventRecord(ev_side_, side_), "event");
  // main stream, after the speculative continuation and the partition: the
  // late statistics
  cuda_check(cudaEventRecord(ev_[1], stream_), "event");
  cuda_check(cudaStreamWaitEvent(stream_, ev_part_, 0), "stream wait");
  if (dcc) {
    cuda_check(launch_dcov_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, d_centre_.get(), d_dcov_.get(),
                                      stream_, late_c),
               "dcov components");
    cuda_check(cudaStreamWaitEvent(stream_, ev_side_, 0), "stream wait");
    cuda_check(launch_dcov_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_dcov_.get(),
                                 d_pairs_.get(), npairs, d_records_.get(), stream_, late_p),
               "dcov pairs");
    cuda_check(cudaEventRecord(ev_[2], stream_), "event");
    cuda_check(launch_guard_select(d_records_.get(), d_pairs_.get(), npairs, ncomp, guard_cap_, kGuardLower,
                                   kGuardUpper, guard, stream_, late_p, 1, mark),
               "guard select");
    cuda_check(launch_legacy_eigen(d_resid_.get(), n, d_comp_cols_.get(), guard, slot_comps, guard_cap_, lr_ctas,
                                   opt_.num_col, d_legacy_ws_.get(), d_lr_vals_.get(), d_lr_vecs_.get(),
                                   d_lr_status_.get(), stream_, mark + 1),
               "legacy eigen");
    cuda_check(launch_legacy_pairs(n, opt_.num_col, d_lr_vals_.get(), d_lr_vecs_.get(), d_dcov_.get(), guard, glist,
                                   comp_slot, d_pairs_.get(), npairs, d_records_.get(), stream_, mark),
               "legacy pairs");
    launches_ += 5;
  } else {
    cuda_check(launch_hsic_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, opt_.num_col, opt_.hsic_sig,
                                      d_factors_.get(), d_hsic_.get(), stream_, late_c),
               "hsic components");
    cuda_check(cudaStreamWaitEvent(stream_, ev_side_, 0), "stream wait");
    cuda_check(launch_hsic_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), d_pairs_.get(), npairs,
                                 d_records_.get(), stream_, late_p),
               "hsic pairs");
    cuda_check(cudaEventRecord(ev_[2], stream_), "event");
    launches_ += 2;
  }
  cuda_check(cudaEventRecord(ev_[3], stream_), "event");
}

void Engine::enqueue_stats_serial() {
  const int n = n_;
  const int ncomp = static_cast<int>(comps_.size());
  const int npairs = static_cast<int>(pairs_.size());
  if (stats_enabled_ && npairs > 0) {
    const int method = opt_.ci_method;
    if (method == FKPC_DCC_GAMMA || method == FKPC_DCC_PERM) {
      cuda_check(launch_dcov_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, d_centre_.get(), d_dcov_.get(),
                                        stream_),
                 "dcov components");
      ++launches_;
    }
    if (method == FKPC_DCC_GAMMA) {
      cuda_check(launch_dcov_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_dcov_.get(),
                                   d_pairs_.get(), npairs, d_records_.get(), stream_),
                 "dcov pairs");
      ++launches_;
      cuda_check(cudaEventRecord(ev_[2], stream_), "event");
      int* guard = d_guard_.get();
      cuda_check(launch_guard_select(d_records_.get(), d_pairs_.get(), npairs, ncomp, guard_cap_, kGuardLower,
                                     kGuardUpper, guard, stream_),
                 "guard select");
      const int* list = guard + 2;
      const int* comp_slot = list + npairs;
      const int* slot_comps = comp_slot + ncomp;
      cuda_check(launch_legacy_eigen(d_resid_.get(), n, d_comp_cols_.get(), guard, slot_comps, guard_cap_,
                                     lowrank_launch_ctas(), opt_.num_col, d_legacy_ws_.get(),
                                     d_lr_vals_.get(), d_lr_vecs_.get(), d_lr_status_.get(), stream_),
                 "legacy eigen");
      cuda_check(launch_legacy_pairs(n, opt_.num_col, d_lr_vals_.get(), d_lr_vecs_.get(), d_dcov_.get(), guard, list,
                                     comp_slot, d_pairs_.get(), npairs, d_records_.get(), stream_),
                 "legacy pairs");
      launches_ += 3;
    } else if (method == FKPC_DCC_PERM) {
      cuda_check(launch_dcc_perm_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_pairs_.get(), npairs,
                                       d_perms_.get(), opt_.permutation_replicates, d_records_.get(), stream_),
                 "dcc perm pairs");
      ++launches_;
    } else {
      cuda_check(launch_hsic_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, opt_.num_col, opt_.hsic_sig,
                                        d_factors_.get(), d_hsic_.get(), stream_),
                 "hsic components");
      ++launches_;
      if (method == FKPC_HSIC_GAMMA) {
        cuda_check(launch_hsic_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), d_pairs_.get(), npairs,
                                     d_records_.get(), stream_),
                   "hsic pairs");
      } else {
        cuda_check(launch_hsic_perm_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), d_pairs_.get(), npairs,
                                          d_perms_.get(), opt_.permutation_replicates, d_records_.get(), stream_),
                   "hsic perm pairs");
      }
      ++launches_;
    }
  }
}

void Engine::execute() {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  const bool perm = opt_.ci_method == FKPC_DCC_PERM || opt_.ci_method == FKPC_HSIC_PERM;
  graph_timed_ = false;
  if (opt_.mode == FKPC_MODE_PLAIN && perm) {
    // one permutation test: its launch sequence without a graph
    cuda_check(configure_fit_kernels(), "kernel attributes");
    cuda_check(configure_stat_kernels(n_), "kernel attributes");
    enqueue();
    return;
  }
  if (opt_.mode == FKPC_MODE_PLAIN) {
    // the plain per-test form: each test's own launch set, synchronised
    cuda_check(configure_fit_kernels(), "kernel attributes");
    cuda_check(configure_stat_kernels(n_), "kernel attributes");
    cuda_check(cudaEventRecord(ev_[0], stream_), "event");
    launches_ = 0;
    for (int t = 0; t < static_cast<int>(pairs_.size()); ++t) {
      enqueue_plain_test(t);
      cuda_check(cudaStreamSynchronize(stream_), "plain test");
    }
    cuda_check(cudaEventRecord(ev_[1], stream_), "event");
    cuda_check(cudaEventRecord(ev_[2], stream_), "event");
    cuda_check(cudaEventRecord(ev_[3], stream_), "event");
    return;
  }
  if (!graph_exec_) {
    cuda_check(configure_fit_kernels(), "kernel attributes");
    cuda_check(configure_stat_kernels(n_), "kernel attributes");
    cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      enqueue();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cuda_check(cudaStreamEndCapture(stream_, &graph_), "end capture");
    cuda_check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
  }
  cuda_check(cudaEventRecord(ev_[4], stream_), "event");
  cuda_check(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
  cuda_check(cudaEventRecord(ev_[5], stream_), "event");
  graph_timed_ = true;
}

void Engine::collect(fkpc_ci_record* out, fkpc_stage_stats* stats) {
  auto t0 = std::chrono::steady_clock::now();
  cuda_check(cudaStreamSynchronize(stream_), "batch execution");
  check_geometry();
  std::vector<FitResult> sres(single_jobs_.size()), mres(multi_jobs_.size());
  if (!sres.empty())
    cuda_check(cudaMemcpy(sres.data(), d_single_res_.get(), sres.size() * sizeof(FitResult), cudaMemcpyDeviceToHost), "download");
  if (!mres.empty())
    cuda_check(cudaMemcpy(mres.data(), d_multi_res_.get(), mres.size() * sizeof(FitResult), cudaMemcpyDeviceToHost), "download");
  auto fit_failure = [&](const FitJob& job, const FitResult& r) {
    const Design& des = *designs_[job.design];
    std::string s = "residual fit of variable " + std::to_string(job.column) + " on S = {";
    for (size_t i = 0; i < des.S.size(); ++i) s += (i ? "," : "") + std::to_string(des.S[i]);
    s += "} failed with status " + std::to_string(r.status);
    return Error(r.status == kStatusRank ? FKPC_STATUS_RANK
                                          : (r.status == kStatusNotConverged ? FKPC_STATUS_NOT_CONVERGED : FKPC_STATUS_NUMERIC),
                 s);
  };
  d2h_bytes_ += static_cast<double>((sres.size() + mres.size()) * sizeof(FitResult));
  account_flops(sres, mres);
  collected_ = true;
  // a regression batch reports each fit's status (its residual is NaN); a
  // CI batch fails as a whole
  if (stats_enabled_) {
    for (size_t i = 0; i < sres.size(); ++i)
      if (sres[i].status != kStatusOk) throw fit_failure(single_jobs_[i], sres[i]);
    for (size_t i = 0; i < mres.size(); ++i)
      if (mres[i].status != kStatusOk) throw fit_failure(multi_jobs_[i], mres[i]);
  }
  std::vector<RecordDev> recs(pairs_.size());
  if (!recs.empty() && stats_enabled_)
    cuda_check(cudaMemcpy(recs.data(), d_records_.get(), recs.size() * sizeof(RecordDev), cudaMemcpyDeviceToHost), "download");
  d2h_bytes_ += static_cast<double>(recs.size() * sizeof(RecordDev));
  int guarded = 0;
  if (stats_enabled_ && opt_.ci_method == FKPC_DCC_GAMMA && !pairs_.empty()) {
    int counts[2] = {0, 0};
    cuda_check(cudaMemcpy(counts, d_guard_.get(), sizeof(counts), cudaMemcpyDeviceToHost), "download");
    guarded = counts[0];
    if (counts[1] > guard_cap_) throw Error(FKPC_STATUS_ALLOCATION, "guard-band low-rank capacity exceeded");
    const int slots = std::min(counts[1], guard_cap_);
    std::vector<int> lrs(slots), steps(slots);
    if (slots > 0) {
      cuda_check(cudaMemcpy(lrs.data(), d_lr_status_.get(), slots * sizeof(int), cudaMemcpyDeviceToHost), "download");
      cuda_check(cudaMemcpy(steps.data(), d_lr_status_.get() + guard_cap_, slots * sizeof(int), cudaMemcpyDeviceToHost),
                 "download");
    }
    lowrank_steps_mean_ = 0.0;
    lowrank_steps_max_ = 0;
    for (int k = 0; k < slots; ++k) {
      lowrank_steps_mean_ += steps[k];
      lowrank_steps_max_ = std::max(lowrank_steps_max_, steps[k]);
    }
    if (slots > 0) lowrank_steps_mean_ /= slots;
    lowrank_slots_ = slots;
    for (int s : lrs)
      if (s != kStatusOk) throw Error(FKPC_STATUS_NOT_CONVERGED, "low-rank eigen-solve of a guarded component did not converge");
  }
  double download_ms = ms_since(t0);
  if (out) {
    // a test whose residual came from a rank-truncated fit says so
    std::vector<char> truncated(comps_.size(), 0);
    for (size_t i = 0; i < sres.size(); ++i)
      if (sres[i].flags & kFitFlagRankTruncated) truncated[single_jobs_[i].out] = 1;
    for (size_t i = 0; i < mres.size(); ++i)
      if (mres[i].flags & kFitFlagRankTruncated) truncated[multi_jobs_[i].out] = 1;
    for (size_t t = 0; t < recs.size(); ++t) {
      const RecordDev& r = recs[t];
      fkpc_ci_record& o = out[t];
      o.p_value = r.p_value;
      o.p_exact = r.p_exact;
      o.statistic = r.statistic;
      o.mean = r.mean;
      o.variance = r.variance;
      o.status = r.status;
      o.flags = r.flags | (tests_[t].S.empty() ? FKPC_FLAG_DIRECT : 0u);
      if (t < pairs_.size() && (truncated[pairs_[t].left] || truncated[pairs_[t].right]))
        o.flags |= FKPC_FLAG_RANK_TRUNCATED;
      if (r.status != kStatusOk)
        throw Error(r.status == kStatusNotConverged ? FKPC_STATUS_NOT_CONVERGED : FKPC_STATUS_NUMERIC,
                    "statistic of test " + std::to_string(t) + " failed with status " + std::to_string(r.status));
    }
  }
  if (stats) {
    // stage split from the event pairs of a direct (uncaptured) launch; a graph
    // replay reports its whole device time as fit_ms + statistic_ms = device_ms
    float f_ms = 0.f, s_ms = 0.f, g_ms = 0.f, tot = 0.f;
    if (graph_timed_) {
      cudaEventElapsedTime(&tot, ev_[4], ev_[5]);
    } else {
      cudaEventElapsedTime(&f_ms, ev_[0], ev_[1]);
      cudaEventElapsedTime(&tot, ev_[0], ev_[3]);
      s_ms = tot - f_ms;
      if (stats_enabled_ && opt_.ci_method == FKPC_DCC_GAMMA && !pairs_.empty()) {
        cudaEventElapsedTime(&g_ms, ev_[2], ev_[3]);
        s_ms -= g_ms;
      }
    }
    stats->device_ms = tot;
    stats->setup_ms = setup_ms_;
    stats->upload_ms = upload_ms_;
    stats->fit_ms = f_ms;
    stats->statistic_ms = s_ms;
    stats->refine_ms = g_ms;
    stats->download_ms = download_ms;
    stats->designs = static_cast<int>(sets_.size());
    stats->designs_built = designs_built_;
    stats->smooths_built = smooths_built_;
    stats->plan_ms = call_timed_ ? plan_ms_ : 0.0;
    stats->tprs_host_ms = call_timed_ ? tprs_host_ms_ : 0.0;
    stats->design_host_ms = call_timed_ ? design_host_ms_ : 0.0;
    stats->smooth_wait_ms = call_timed_ ? smooth_wait_ms_ : 0.0;
    stats->late_wait_ms = call_timed_ ? late_wait_ms_ : 0.0;
    float pre = 0.f;
    if (call_timed_) cudaEventElapsedTime(&pre, ev_call_, ev_[0]);
    stats->prefit_device_ms = pre;
    stats->targets = static_cast<int>(single_jobs_.size() + multi_jobs_.size());
    stats->pairs = static_cast<int>(pairs_.size());
    stats->guarded = guarded;
    stats->kernel_launches = launches_;
    stats->h2d_bytes = h2d_bytes_;
    stats->d2h_bytes = d2h_bytes_;
    double evals = 0.0;
    for (const auto& r : sres) evals += r.evaluations;
    for (const auto& r : mres) evals += r.evaluations;
    stats->fit_evaluations = evals;
    stats->fit_flops = stage_flops_[0] + stage_flops_[1] + stage_flops_[2] + stage_flops_[9] + stage_flops_[10];
    double its = 0.0;
    for (const auto& r : sres) its += r.iterations;
    for (const auto& r : mres) its += r.iterations;
    stats->fit_iterations = its;
    stats->lowrank_components = lowrank_slots_;
    stats->lowrank_steps_mean = lowrank_steps_mean_;
    stats->lowrank_steps_max = lowrank_steps_max_;
    stats->statistic_flops = stage_flops_[3] + stage_flops_[4] + stage_flops_[5] + stage_flops_[6];
  }
}

// Algorithmic FP64 flop counts (FMA = 2):
//  fits       : per fit 6nq + E (16 q^3 + 2 m q^3) (comment in the body).
//  dCov components : row sums 2 n^2, squared centred entries 2.5 n (n - 1).
//  dCov pairs      : 4 n (n - 1) (n(n-1)/2 entries x 2 abs-diffs, 4 centring
//                    subtractions and one FMA).
//  HSIC components : per incomplete-Cholesky step k, n exponentials (20 each)
//                    and 2 n k; then 2 n r^2 for |Gc'Gc|_F^2.
//  HSIC pairs      : 2 n rx ry.
void Engine::account_flops(const std::vector<FitResult>& sres, const std::vector<FitResult>& mres) {
  for (double& f : stage_flops_) f = 0.0;
  const double n = n_;
  // The fit stages count the path's algorithmic FP64 work as the scope table
  // of the hot path defines it, per fit: Q'y (4nq) and the residual (2nq),
  // plus 16q^3 (the SVD of the stacked system with U1) + 2mq^3 (the
  // derivatives) per GCV evaluation, E evaluations from the search's own
  // counter.  The kernels execute less (the spectral single-penalty form,
  // the Householder fold, derivatives only at accepted points).
  for (size_t i = 0; i < single_jobs_.size(); ++i) {
    const double q = designs_[single_jobs_[i].design]->q;
    stage_flops_[0] += 6.0 * n * q + (16.0 + 2.0) * q * q * q * sres[i].evaluations;
  }
  for (size_t i = 0; i < multi_jobs_.size(); ++i) {
    const Design& des = *designs_[multi_jobs_[i].design];
    const double q = des.q;
    double rs = 0.0;
    for (int r : des.ranks) rs += r;
    const double f = 6.0 * n * q + (16.0 + 2.0 * des.m) * q * q * q * mres[i].evaluations;
    const bool small = des.q <= kWarpQ && rs <= kWarpR && des.m <= kWarpM;
    const bool large = !small && des.q <= 76 && rs <= 64 && des.m <= kCtaPenalties;
    const bool huge = !small && !large && des.q <= 112 && rs <= 96 && des.m <= kCtaPenalties;
    stage_flops_[small ? 1 : (large ? 2 : (huge ? 9 : 10))] += f;
  }
  if (stats_enabled_) {
    const double nc = static_cast<double>(comps_.size()), np = static_cast<double>(pairs_.size());
    if (opt_.ci_method == FKPC_DCC_GAMMA || opt_.ci_method == FKPC_DCC_PERM) {
      stage_flops_[3] = nc * (2.0 * n * n + 2.5 * n * (n - 1.0));
      const double reps = opt_.ci_method == FKPC_DCC_PERM ? opt_.permutation_replicates + 1.0 : 1.0;
      stage_flops_[4] = np * reps * 4.0 * n * (n - 1.0);
    }
    if (opt_.ci_method == FKPC_HSIC_GAMMA || opt_.ci_method == FKPC_HSIC_PERM) {
      const double r = opt_.num_col;
      stage_flops_[5] = nc * (r * n * 20.0 + n * r * r + 2.0 * n * r * r);
      const double reps = opt_.ci_method == FKPC_HSIC_PERM ? opt_.permutation_replicates + 1.0 : 1.0;
      stage_flops_[6] = np * reps * 2.0 * n * r * r;
    }
  }
}

void Engine::enqueue_plain_test(int t) {
  const int n = n_;
  const int ncomp = static_cast<int>(comps_.size());
  const int npairs = static_cast<int>(pairs_.size());
  const int d0 = plain_direct_off_[t], d1 = plain_direct_off_[t + 1];
  if (d1 > d0) {
    dim3 grid((n + 255) / 256, static_cast<unsigned>(d1 - d0));
    gather_columns_kernel<<<grid, 256, 0, stream_>>>(d_data_.get(), n, d_direct_cols_.get() + d0,
                                                      d_direct_slots_.get() + d0, d1 - d0, d_resid_.get());
    cuda_check(cudaGetLastError(), "gather columns");
    ++launches_;
  }
  const int s0 = plain_single_off_[t], s1 = plain_single_off_[t + 1];
  if (s1 > s0) {
    cuda_check(launch_fit_single(d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_single_jobs_.get() + s0, s1 - s0,
                                 d_resid_.get(), d_single_res_.get() + s0, stream_),
               "fit single");
    ++launches_;
  }
  const int a0 = plain_small_off_[t], a1 = plain_small_off_[t + 1];
  if (a1 > a0) {
    cuda_check(launch_fit_multi(0, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_small_.get() + a0, a1 - a0, d_resid_.get(), d_multi_res_.get(), stream_, opt_.selection),
               "fit multi");
    ++launches_;
  }
  const int b0 = plain_large_off_[t], b1 = plain_large_off_[t + 1];
  if (b1 > b0) {
    cuda_check(launch_fit_multi(1, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_large_.get() + b0, b1 - b0, d_resid_.get(), d_multi_res_.get(), stream_, opt_.selection),
               "fit multi");
    ++launches_;
  }
  const int h0 = plain_huge_off_[t], h1 = plain_huge_off_[t + 1];
  if (h1 > h0) {
    cuda_check(launch_fit_multi(2, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_huge_.get() + h0, h1 - h0, d_resid_.get(), d_multi_res_.get(), stream_,
                                opt_.selection, d_fit_ws_.get()),
               "fit multi");
    ++launches_;
  }
  const int w0 = plain_wide_off_[t], w1 = plain_wide_off_[t + 1];
  if (w1 > w0) {
    cuda_check(launch_fit_multi(3, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                d_multi_wide_.get() + w0, w1 - w0, d_resid_.get(), d_multi_res_.get(), stream_,
                                opt_.selection, d_fit_ws_.get(), nullptr, nullptr, nullptr, nullptr, 0,
                                d_wide_log_sp_.get() + static_cast<size_t>(w0) * kMaxPenalties),
               "fit multi");
    ++launches_;
  }
  const int method = opt_.ci_method;
  const PairJob* pair = d_pairs_.get() + t;
  const int* cols = d_comp_cols_.get() + 2 * t;
  if (method == FKPC_DCC_GAMMA) {
    // the two components of test t are 2t and 2t+1 (no sharing in this form)
    cuda_check(launch_dcov_components(d_resid_.get(), n, cols, 2, d_centre_.get() + static_cast<size_t>(n) * 2 * t,
                                      d_dcov_.get() + 2 * t, stream_),
               "dcov components");
    cuda_check(launch_dcov_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_dcov_.get(), pair, 1,
                                 d_records_.get(), stream_),
               "dcov pairs");
    int* guard = d_guard_.get();
    cuda_check(launch_guard_select(d_records_.get(), pair, 1, ncomp, guard_cap_, kGuardLower, kGuardUpper, guard, stream_),
               "guard select");
    cuda_check(launch_legacy_eigen(d_resid_.get(), n, d_comp_cols_.get(), guard, guard + 2 + 1 + ncomp, guard_cap_, 2,
                                   opt_.num_col, d_legacy_ws_.get(), d_lr_vals_.get(), d_lr_vecs_.get(),
                                   d_lr_status_.get(), stream_),
               "legacy eigen");
    cuda_check(launch_legacy_pairs(n, opt_.num_col, d_lr_vals_.get(), d_lr_vecs_.get(), d_dcov_.get(), guard, guard + 2,
                                   guard + 2 + 1, pair, 1, d_records_.get(), stream_),
               "legacy pairs");
    launches_ += 5;
  } else if (method == FKPC_HSIC_GAMMA) {
    cuda_check(launch_hsic_components(d_resid_.get(), n, cols, 2, opt_.num_col, opt_.hsic_sig,
                                      d_factors_.get() + static_cast<size_t>(n) * opt_.num_col * 2 * t,
                                      d_hsic_.get() + 2 * t, stream_),
               "hsic components");
    cuda_check(launch_hsic_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), pair, 1, d_records_.get(), stream_),
               "hsic pairs");
    launches_ += 2;
  } else {
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "the plain form covers the gamma methods; permutation tests run batched");
  }
  (void)npairs;
}

double Engine::execute_timed(int repeats) {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  if (opt_.mode == FKPC_MODE_PLAIN) {
    cuda_check(configure_fit_kernels(), "kernel attributes");
    cuda_check(configure_stat_kernels(n_), "kernel attributes");
    float total = 0.f;
    for (int r = 0; r < repeats; ++r) {
      cuda_check(cudaEventRecord(ev_[4], stream_), "event");
      execute();
      cuda_check(cudaEventRecord(ev_[5], stream_), "event");
      cuda_check(cudaEventSynchronize(ev_[5]), "event sync");
      float ms = 0.f;
      cuda_check(cudaEventElapsedTime(&ms, ev_[4], ev_[5]), "event time");
      total += ms;
    }
    return total;
  }
  execute();  // builds the graph on first use
  cuda_check(cudaStreamSynchronize(stream_), "warm graph");
  cuda_check(cudaEventRecord(ev_[4], stream_), "event");
  for (int r = 0; r < repeats; ++r) cuda_check(cudaGraphLaunch(graph_exec_, stream_), "graph launch");
  cuda_check(cudaEventRecord(ev_[5], stream_), "event");
  cuda_check(cudaEventSynchronize(ev_[5]), "event sync");
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, ev_[4], ev_[5]), "event time");
  return ms;
}

double Engine::time_stage(int stage, int repeats, double* flops_per_launch) {
  if (!collected_) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "collect the prepared batch before timing a stage");
  if (stage < 0 || stage > 10) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "unknown stage");
  cuda_check(configure_fit_kernels(), "kernel attributes");
  cuda_check(configure_stat_kernels(n_), "kernel attributes");
  const int n = n_;
  const int ncomp = static_cast<int>(comps_.size());
  const int npairs = static_cast<int>(pairs_.size());
  int* guard = d_guard_.get();
  auto launch = [&]() -> cudaError_t {
    switch (stage) {
      case 0: return launch_fit_single(d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_single_jobs_.get(),
                                       static_cast<int>(single_jobs_.size()), d_resid_.get(), d_single_res_.get(), stream_);
      case 1: return launch_fit_multi(0, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                      d_multi_small_.get(), static_cast<int>(multi_small_.size()), d_resid_.get(),
                                      d_multi_res_.get(), stream_, opt_.selection, nullptr, d_fit_states_.get(),
                                      d_defer_list_.get(), d_defer_count_.get(), nullptr,
                                      tuning_.defer_evaluations);
      case 2: return launch_fit_multi(1, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                      d_multi_large_.get(), static_cast<int>(multi_large_.size()), d_resid_.get(),
                                      d_multi_res_.get(), stream_, opt_.selection);
      case 9: return launch_fit_multi(2, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                      d_multi_huge_.get(), static_cast<int>(multi_huge_.size()), d_resid_.get(),
                                      d_multi_res_.get(), stream_, opt_.selection, d_fit_ws_.get());
      case 10: return launch_fit_multi(3, d_designs_.get(), d_arena_.get(), d_data_.get(), n, d_multi_jobs_.get(),
                                       d_multi_wide_.get(), static_cast<int>(multi_wide_.size()), d_resid_.get(),
                                       d_multi_res_.get(), stream_, opt_.selection, d_fit_ws_.get(), nullptr,
                                       nullptr, nullptr, nullptr, 0, d_wide_log_sp_.get());
      case 3: return launch_dcov_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, d_centre_.get(),
                                            d_dcov_.get(), stream_);
      case 4: return launch_dcov_pairs(d_resid_.get(), n, d_comp_cols_.get(), d_centre_.get(), d_dcov_.get(),
                                       d_pairs_.get(), npairs, d_records_.get(), stream_);
      case 5: return launch_hsic_components(d_resid_.get(), n, d_comp_cols_.get(), ncomp, opt_.num_col, opt_.hsic_sig,
                                            d_factors_.get(), d_hsic_.get(), stream_);
      case 6: return launch_hsic_pairs(n, opt_.num_col, d_factors_.get(), d_hsic_.get(), d_pairs_.get(), npairs,
                                       d_records_.get(), stream_);
      case 7: return launch_legacy_eigen(d_resid_.get(), n, d_comp_cols_.get(), guard, guard + 2 + npairs + ncomp,
                                         guard_cap_, lowrank_launch_ctas(), opt_.num_col,
                                         d_legacy_ws_.get(), d_lr_vals_.get(), d_lr_vecs_.get(), d_lr_status_.get(),
                                         stream_);
      default: return launch_legacy_pairs(n, opt_.num_col, d_lr_vals_.get(), d_lr_vecs_.get(), d_dcov_.get(), guard,
                                          guard + 2, guard + 2 + npairs, d_pairs_.get(), npairs, d_records_.get(),
                                          stream_);
    }
  };
  const bool dcc = opt_.ci_method == FKPC_DCC_GAMMA || opt_.ci_method == FKPC_DCC_PERM;
  const bool hsic = opt_.ci_method == FKPC_HSIC_GAMMA || opt_.ci_method == FKPC_HSIC_PERM;
  if (((stage == 3 || stage == 4) && !dcc) || ((stage == 5 || stage == 6) && !hsic) ||
      ((stage == 7 || stage == 8) && opt_.ci_method != FKPC_DCC_GAMMA))
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "stage not part of the prepared method");
  cuda_check(launch(), "stage warm-up");
  cuda_check(cudaStreamSynchronize(stream_), "stage warm-up");
  cuda_check(cudaEventRecord(ev_[4], stream_), "event");
  for (int r = 0; r < repeats; ++r) cuda_check(launch(), "stage launch");
  cuda_check(cudaEventRecord(ev_[5], stream_), "event");
  cuda_check(cudaEventSynchronize(ev_[5]), "event sync");
  float ms = 0.f;
  cuda_check(cudaEventElapsedTime(&ms, ev_[4], ev_[5]), "event time");
  if (flops_per_launch) *flops_per_launch = stage_flops_[stage];
  return ms / std::max(1, repeats);
}

void Engine::set_tuning(const fkpc_tuning& t) {
  if (t.defer_evaluations < 0 || t.split_statistics < 0 || t.split_statistics > 1 || t.lowrank_ctas_per_sm < 1 ||
      t.lowrank_ctas_per_sm > 4 || t.tprs_ctas_per_sm < 1 || t.tprs_ctas_per_sm > 4)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT,
                "tuning out of range (defer >= 0, split 0/1, Lanczos CTAs per SM 1..4)");
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  cuda_check(cudaStreamSynchronize(stream_), "tuning");
  tuning_ = t;
  release_graph();
  if (lr_ws_ctas_ > 0 && n_ > 0 && lr_ws_ctas_ < legacy_ctas()) {
    // a prepared guard band: its workspace follows the new CTA count
    d_legacy_ws_.ensure(legacy_eigen_workspace_doubles(n_, legacy_ctas()));
    lr_ws_ctas_ = legacy_ctas();
  }
}

double Engine::measure_fp64_peak() {
  cuda_check(cudaSetDevice(device_), "cudaSetDevice");
  int sms = 0;
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "device attribute");
  const int blocks = sms * 8, iters = 4096;
  DevBuf<double> out;
  double* d = out.ensure(static_cast<size_t>(blocks) * 256);
  cuda_check(launch_fp64_peak(d, blocks, iters, stream_), "fp64 probe");
  cuda_check(cudaStreamSynchronize(stream_), "fp64 probe");
  double best = 0.0;
  for (int rep = 0; rep < 5; ++rep) {
    cuda_check(cudaEventRecord(ev_[4], stream_), "event");
    cuda_check(launch_fp64_peak(d, blocks, iters, stream_), "fp64 probe");
    cuda_check(cudaEventRecord(ev_[5], stream_), "event");
    cuda_check(cudaEventSynchronize(ev_[5]), "event sync");
    float ms = 0.f;
    cuda_check(cudaEventElapsedTime(&ms, ev_[4], ev_[5]), "event time");
    const double flops = 2.0 * 16.0 * iters * 256.0 * blocks;
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  return best;
}

void Engine::regress(const std::vector<int>& targets, const std::vector<std::vector<int>>& sets,
                     double* residuals, double* log_sp, int max_penalties, int* status, int selection,
                     int* evaluations) {
  if (targets.size() != sets.size()) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "targets and sets differ in length");
  std::vector<Test> tests;
  for (size_t i = 0; i < targets.size(); ++i) {
    Test t;
    t.x = targets[i];
    t.y = targets[i] == 0 ? 1 : 0;  // placeholder partner; only the x component is read back
    t.S = sets[i];
    for (int s : t.S)
      if (s == t.y) t.y = -1;
    if (t.y < 0)
      for (int c = 0; c < p_; ++c)
        if (c != t.x && std::find(t.S.begin(), t.S.end(), c) == t.S.end()) { t.y = c; break; }
    tests.push_back(t);
  }
  fkpc_options opt;
  fkpc_default_options(&opt);
  opt.selection = selection;
  opt_ = opt;
  call_timed_ = false;
  release_graph();
  cuda_check(cudaStreamSynchronize(stream_), "set-up");
  stage_reset();
  d2h_bytes_ = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  regress_only_ = true;
  try {
    plan_components(tests);
  } catch (...) {
    regress_only_ = false;
    throw;
  }
  regress_only_ = false;
  designs_built_ = 0;
  for (const auto& S : sets_) designs_built_ += cache_->has_design(S) ? 0 : 1;
  smooths_built_ = static_cast<int>(univariate_columns().size());
  build_designs();
  setup_ms_ = ms_since(t0);
  stats_enabled_ = false;
  pack_and_upload(opt, nullptr);
  cuda_check(configure_fit_kernels(), "kernel attributes");
  enqueue();
  cuda_check(cudaStreamSynchronize(stream_), "regress");
  collect(nullptr, nullptr);
  const int n = n_;
  std::vector<double> slab(static_cast<size_t>(n) * comps_.size());
  cuda_check(cudaMemcpy(slab.data(), d_resid_.get(), slab.size() * sizeof(double), cudaMemcpyDeviceToHost), "download");
  std::vector<FitResult> sres(single_jobs_.size()), mres(multi_jobs_.size());
  if (!sres.empty())
    cuda_check(cudaMemcpy(sres.data(), d_single_res_.get(), sres.size() * sizeof(FitResult), cudaMemcpyDeviceToHost), "download");
  if (!mres.empty())
    cuda_check(cudaMemcpy(mres.data(), d_multi_res_.get(), mres.size() * sizeof(FitResult), cudaMemcpyDeviceToHost), "download");
  std::vector<const FitResult*> by_comp(comps_.size(), nullptr);
  for (size_t i = 0; i < single_jobs_.size(); ++i) by_comp[single_jobs_[i].out] = &sres[i];
  for (size_t i = 0; i < multi_jobs_.size(); ++i) by_comp[multi_jobs_[i].out] = &mres[i];
  // the wide class's log(lambda), all m of them, per component
  std::vector<double> wide(multi_wide_.size() * static_cast<size_t>(kMaxPenalties));
  std::vector<const double*> wide_by_comp(comps_.size(), nullptr);
  if (!wide.empty()) {
    cuda_check(cudaMemcpy(wide.data(), d_wide_log_sp_.get(), wide.size() * sizeof(double), cudaMemcpyDeviceToHost),
               "download");
    for (size_t k = 0; k < multi_wide_.size(); ++k)
      wide_by_comp[multi_jobs_[multi_wide_[k]].out] = wide.data() + k * kMaxPenalties;
  }
  for (size_t i = 0; i < targets.size(); ++i) {
    const int c = pairs_[i].left;
    std::copy(slab.begin() + static_cast<size_t>(n) * c, slab.begin() + static_cast<size_t>(n) * (c + 1),
              residuals + static_cast<size_t>(n) * i);
    const FitResult* r = by_comp[c];
    const double* wl = wide_by_comp[c];
    if (status) status[i] = r ? r->status : kStatusOk;
    if (evaluations) evaluations[i] = r ? r->evaluations : 0;
    if (log_sp)
      for (int j = 0; j < max_penalties; ++j)
        log_sp[i * static_cast<size_t>(max_penalties) + j] =
            wl ? (j < kMaxPenalties ? wl[j] : NAN) : ((r && j < kCtaPenalties) ? r->log_sp[j] : NAN);
  }
  stats_enabled_ = true;
}

void Engine::adjoint(int target, const std::vector<int>& S, int count, const double* rho, double* score,
                     double* grad, double* gn_hessian, double* exact_hessian) {
  if (S.size() < 3) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "the GCV adjoint covers additive designs (|S| >= 3)");
  if (target < 0 || target >= p_) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "target column out of range");
  for (size_t i = 0; i < S.size(); ++i) {
    if (S[i] < 0 || S[i] >= p_ || S[i] == target) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "invalid conditioning set");
    for (size_t j = 0; j < i; ++j)
      if (S[j] == S[i]) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "repeated conditioning variable");
  }
  if (count < 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "negative point count");
  Test t;
  t.x = target;
  t.y = -1;  // a partner column outside {target} and S; only the target's fit is used
  for (int c = 0; c < p_ && t.y < 0; ++c)
    if (c != target && std::find(S.begin(), S.end(), c) == S.end()) t.y = c;
  if (t.y < 0) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "no column outside the target and S");
  t.S = S;
  fkpc_options opt;
  fkpc_default_options(&opt);
  opt_ = opt;
  release_graph();
  cuda_check(cudaStreamSynchronize(stream_), "set-up");
  stage_reset();
  d2h_bytes_ = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  plan_components({t});
  build_designs();
  setup_ms_ = ms_since(t0);
  stats_enabled_ = false;
  pack_and_upload(opt, nullptr);
  stats_enabled_ = true;
  cuda_check(configure_fit_kernels(), "kernel attributes");
  const Design& des = *designs_.at(0);
  const int m = des.m;
  int rsum = 0;
  for (int r : des.ranks) rsum += r;
  if (des.q > 112 || rsum > 96 || m > kCtaPenalties)
    throw Error(FKPC_STATUS_INVALID_ARGUMENT, "the GCV adjoint covers designs with |S| <= 12 (q <= 112)");
  const int qclass = (des.q <= kWarpQ && rsum <= kWarpR && m <= kWarpM) ? 0 : (des.q <= 76 && rsum <= 64 ? 1 : 2);
  if (count == 0) return;
  DevBuf<double> d_rho, d_score, d_grad, d_gn, d_hess;
  if (qclass == 2) d_fit_ws_.ensure(multi_workspace_doubles(2, count));
  DevBuf<int> d_status;
  const size_t cm = static_cast<size_t>(count) * m, cmm = cm * m;
  cuda_check(cudaMemcpyAsync(d_rho.ensure(cm), rho, cm * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload");
  cuda_check(launch_gcv_adjoint(qclass, d_designs_.get(), 0, d_arena_.get(), d_data_.get() + static_cast<size_t>(n_) * target,
                                n_, d_rho.get(), count, d_score.ensure(count), d_grad.ensure(cm), d_gn.ensure(cmm),
                                d_hess.ensure(cmm), d_status.ensure(count), stream_, qclass == 2 ? d_fit_ws_.get() : nullptr),
             "gcv adjoint");
  ++launches_;
  std::vector<int> st(count);
  cuda_check(cudaMemcpyAsync(st.data(), d_status.get(), count * sizeof(int), cudaMemcpyDeviceToHost, stream_), "download");
  if (score)
    cuda_check(cudaMemcpyAsync(score, d_score.get(), count * sizeof(double), cudaMemcpyDeviceToHost, stream_), "download");
  if (grad) cuda_check(cudaMemcpyAsync(grad, d_grad.get(), cm * sizeof(double), cudaMemcpyDeviceToHost, stream_), "download");
  if (gn_hessian)
    cuda_check(cudaMemcpyAsync(gn_hessian, d_gn.get(), cmm * sizeof(double), cudaMemcpyDeviceToHost, stream_), "download");
  if (exact_hessian)
    cuda_check(cudaMemcpyAsync(exact_hessian, d_hess.get(), cmm * sizeof(double), cudaMemcpyDeviceToHost, stream_),
               "download");
  cuda_check(cudaStreamSynchronize(stream_), "gcv adjoint");
  for (int k = 0; k < count; ++k)
    if (st[k] != kStatusOk)
      throw Error(st[k] == kStatusRank ? FKPC_STATUS_RANK : FKPC_STATUS_NUMERIC,
                  "GCV evaluation failed at point " + std::to_string(k));
}

void Engine::statistics(const double* residuals, int m, const std::vector<int>& left, const std::vector<int>& right,
                        const int* permutations, const fkpc_options& opt, fkpc_ci_record* out) {
  const int n = n_;
  if (left.size() != right.size()) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "left and right differ in length");
  for (size_t i = 0; i < left.size(); ++i)
    if (left[i] < 0 || left[i] >= m || right[i] < 0 || right[i] >= m)
      throw Error(FKPC_STATUS_INVALID_ARGUMENT, "residual column index out of range");
  opt_ = opt;
  call_timed_ = false;
  release_graph();
  tests_.clear();
  comps_.assign(m, Component{0, -1});
  pairs_.clear();
  for (size_t i = 0; i < left.size(); ++i) {
    pairs_.push_back(PairJob{left[i], right[i], static_cast<int>(i), 0});
    tests_.push_back(Test{left[i], right[i], {}});
  }
  sets_.clear();
  designs_.clear();
  single_jobs_.clear();
  multi_jobs_.clear();
  multi_small_.clear();
  multi_large_.clear();
  multi_huge_.clear();
  multi_wide_.clear();
  direct_cols_.clear();
  direct_slots_.clear();
  stats_enabled_ = true;
  // pack: no designs; residual slab = caller residuals
  std::vector<int> ident(m);
  for (int c = 0; c < m; ++c) ident[c] = c;
  upload(d_comp_cols_, ident, stream_);
  upload(d_pairs_, pairs_, stream_);
  double* slab = d_resid_.ensure(static_cast<size_t>(n) * m);
  cuda_check(cudaMemcpyAsync(slab, residuals, sizeof(double) * n * static_cast<size_t>(m), cudaMemcpyHostToDevice, stream_),
             "upload residuals");
  d_records_.ensure(pairs_.size());
  const size_t ncomp = static_cast<size_t>(m), npairs = pairs_.size();
  late_designs_ = false;
  d_late_col_.ensure(ncomp);
  d_part_.ensure(4 + 2 * ncomp + 2 * npairs);
  d_guard_mark_.ensure(2);
  if (opt.ci_method == FKPC_DCC_GAMMA || opt.ci_method == FKPC_DCC_PERM) {
    d_centre_.ensure(static_cast<size_t>(n) * ncomp);
    d_dcov_.ensure(ncomp);
  }
  if (opt.ci_method == FKPC_HSIC_GAMMA || opt.ci_method == FKPC_HSIC_PERM) {
    d_factors_.ensure(static_cast<size_t>(n) * opt.num_col * ncomp);
    d_hsic_.ensure(ncomp);
  }
  if (opt.ci_method == FKPC_DCC_GAMMA) {
    guard_cap_ = static_cast<int>(ncomp);
    d_guard_.ensure(2 + npairs + ncomp + guard_cap_);
    d_lr_vals_.ensure(static_cast<size_t>(guard_cap_) * opt.num_col);
    d_lr_vecs_.ensure(static_cast<size_t>(guard_cap_) * opt.num_col * n);
    d_lr_status_.ensure(2 * static_cast<size_t>(guard_cap_));
    d_legacy_ws_.ensure(legacy_eigen_workspace_doubles(n, legacy_ctas()));
      lr_ws_ctas_ = legacy_ctas();
  }
  if (opt.ci_method == FKPC_DCC_PERM || opt.ci_method == FKPC_HSIC_PERM) {
    if (!permutations) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation methods need a permutation table");
    const size_t cnt = npairs * static_cast<size_t>(opt.permutation_replicates) * n;
    for (size_t i = 0; i < cnt; ++i)
      if (permutations[i] < 0 || permutations[i] >= n) throw Error(FKPC_STATUS_INVALID_ARGUMENT, "permutation entry out of range");
    int* d = d_perms_.ensure(cnt);
    cuda_check(cudaMemcpyAsync(d, permutations, cnt * sizeof(int), cudaMemcpyHostToDevice, stream_), "upload perms");
  }
  cuda_check(configure_stat_kernels(n), "kernel attributes");
  enqueue();
  collect(out, nullptr);
}

}  // namespace fkpc
