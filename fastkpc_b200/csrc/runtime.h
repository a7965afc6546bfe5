// Batched CI-test engine: host-side batching of one level's tests into
// designs, residual components and pairs; device arena packing; a fixed
// launch sequence captured once as a CUDA graph and replayed.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fastkpc_b200.h"
#include "design.h"
#include "device.h"
#include "kernels.h"
#include "rstream.h"

namespace fkpc {

struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);

template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (ptr_) cudaFree(ptr_);
  }
  T* ensure(size_t count) {
    if (count == 0) count = 1;
    if (count > cap_) {
      if (ptr_) cudaFree(ptr_);
      ptr_ = nullptr;
      cap_ = 0;
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr_), count * sizeof(T));
      if (e != cudaSuccess) {
        ptr_ = nullptr;
        throw Error(FKPC_STATUS_ALLOCATION, std::string("device allocation failed: ") + cudaGetErrorString(e));
      }
      cap_ = count;
    }
    return ptr_;
  }
  T* get() const { return ptr_; }
  size_t capacity() const { return cap_; }

 private:
  T* ptr_ = nullptr;
  size_t cap_ = 0;
};

struct Test {
  int x, y;
  std::vector<int> S;
};

struct Component {
  int target;
  int design;  // -1 for a direct (|S| = 0) component
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  void load(const double* data, int n, int p);
  int n() const { return n_; }
  int p() const { return p_; }

  // Batched form: plan, set-up, pack and upload one batch of tests.
  void prepare(const std::vector<Test>& tests, const fkpc_options& opt, RStream* stream);
  // One-shot batched form (prepare + execute without a graph): the device
  // work that needs no bivariate basis -- the additive geometry and the
  // multi-penalty fits -- is queued right behind the bivariate thin-plate
  // kernels, while the host finishes those bases; collect() follows.
  void run_batch(const std::vector<Test>& tests, const fkpc_options& opt, RStream* stream);
  // Enqueue the device work of the prepared batch (CUDA graph replay).
  void execute();
  // Wait, copy results back and validate statuses.
  void collect(fkpc_ci_record* out, fkpc_stage_stats* stats);

  // Residual fits only (the regrXonS stage).
  void regress(const std::vector<int>& targets, const std::vector<std::vector<int>>& sets,
               double* residuals, double* log_sp, int max_penalties, int* status,
               int selection = FKPC_SELECT_MAGIC, int* evaluations = nullptr);
  // The device thin-plate set-up of the bivariate smooth on {a, b} alone:
  // its k = 30 Ritz values (descending) and vectors (nu x 30, normalised,
  // largest-magnitude entry positive).  path: 2 block Lanczos, 1
  // single-vector, 0 not taken by the device (too few or too many unique
  // locations); ok: the Ritz pairs converged.
  void tprs_export(int a, int b, int* nu, int* path, int* ok, std::vector<double>* vals, std::vector<double>* U);
  // Statistics only, on caller residual columns.
  void statistics(const double* residuals, int m, const std::vector<int>& left, const std::vector<int>& right,
                  const int* permutations, const fkpc_options& opt, fkpc_ci_record* out);
  // GCV score, gradient, Gauss-Newton and exact Hessian in log(lambda) of the
  // additive fit of column ``target`` on S at ``count`` points (rho: count x m).
  void adjoint(int target, const std::vector<int>& S, int count, const double* rho, double* score, double* grad,
               double* gn_hessian, double* exact_hessian);
  // Repeated graph launches of the prepared batch, timed with CUDA events.
  double execute_timed(int repeats);
  // One kernel of the prepared batch replayed alone: mean ms per launch.
  double time_stage(int stage, int repeats, double* flops_per_launch);
  double measure_fp64_peak();
  fkpc_tuning tuning() const { return tuning_; }
  void set_tuning(const fkpc_tuning& t);  // validates; the next execution re-captures its graph
  cudaStream_t stream() const { return stream_; }
  // When set, packing a permutation batch appends the stream's state after
  // each test's permutations (a speculative caller rolls back to one).
  void set_stream_snapshots(std::vector<RStream>* s) { stream_snapshots_ = s; }
  int launches() const { return launches_; }
  // changes with every load(): a session checks that its data is still loaded
  uint64_t load_id() const { return load_id_; }
  double setup_ms() const { return setup_ms_; }

 private:
  void plan_components(const std::vector<Test>& tests);
  void enqueue_plain_test(int t);  // one test's launch set (plain form)
  double execute_plain_timed(int repeats);
  void build_designs();
  void build_univariate_smooths();
  // copies made while earlier stream work may still run go through page-locked
  // staging: a copy from pageable memory would first wait for the whole stream.
  // A bump allocator over a persistent buffer; a full buffer is retired (kept
  // until the next reset) and replaced by a larger one.  stage_reset() only
  // when nothing on the stream reads staged memory.
  void stage_reset();
  void* stage_alloc(size_t bytes);
  template <class T>
  double stage_upload(DevBuf<T>& buf, const std::vector<T>& host, cudaStream_t st = nullptr);
  void enqueue_multi();  // the multi-penalty fit classes
  // direct columns, single-penalty fits, statistics.  For the gamma methods
  // the single-penalty fits and the statistics of every pair whose residuals
  // are final once the one-warp fit kernel has run go to the side stream
  // (early), beside the speculative continuation; the pairs of the fits it
  // continues follow on the main stream (late).
  void enqueue_rest();
  void enqueue_stats_serial();  // every statistic on the main stream, after every fit
  // pending bivariate designs: descriptors, geometry, on stream ``st``
  // (the side stream uploads the descriptor array to its own buffer)
  void pack_late(cudaStream_t st);
  bool split_stats() const;  // the early / late statistic split applies
  void check_geometry();  // statuses of the geometry kernels (after a synchronisation)
  // one level's thin-plate smooths (dim 2: bivariate, dim 1: univariate) on
  // the device, in flight
  struct TprsBatch {
    int dim = 2;
    std::vector<std::vector<int>> sets;
    std::vector<TprsPrep> preps;
    std::vector<size_t> idx;  // sets taken by the device
    std::vector<int> nus;
    const double* X = nullptr;  // device: design c's basis at X + c n k (smooth store)
    double* S = nullptr;        // page-locked results (inside the staging arena)
    double* colsq = nullptr;
    int* status = nullptr;
  };
  // on stream st with ctas_per_sm Lanczos CTAs per SM
  void launch_tprs_batch(const std::vector<std::vector<int>>& sets, int dim, TprsBatch* batch, cudaStream_t st,
                         int ctas_per_sm);
  void finish_tprs_batch(TprsBatch* batch);
  std::vector<std::vector<int>> univariate_columns();  // variables whose smooth the cache lacks
  template <class Pick>
  void build_host_designs(Pick pick);
  // defer: leave the stream running (the geometry statuses are checked by collect)
  void pack_and_upload(const fkpc_options& opt, RStream* stream, bool defer = false);
  void enqueue();  // the launch sequence
  void release_graph();
  double* pinned_arena(size_t count);  // persistent page-locked staging buffer of the design arena

  int device_ = 0;
  int sms_ = 148;
  fkpc_tuning tuning_{25, 1, 2, 2};
  int legacy_ctas() const { return tuning_.lowrank_ctas_per_sm * sms_; }
  int lr_ws_ctas_ = 0;  // CTAs the guard-band workspace was sized for
  // guard-band Lanczos CTAs of a launch: never more than the workspace holds
  int lowrank_launch_ctas() const { return std::min(std::min(legacy_ctas(), guard_cap_), lr_ws_ctas_); }
  cudaStream_t stream_ = nullptr;
  cudaStream_t side_ = nullptr;  // early statistics beside the speculative continuation
  cudaEvent_t ev_warp_ = nullptr;  // main stream: every fit but the continued ones is done
  cudaEvent_t ev_side_ = nullptr;  // side stream: the early statistics are done
  cudaEvent_t ev_part_ = nullptr;  // side stream: the early / late lists are written
  int n_ = 0, p_ = 0;
  std::vector<double> host_data_;
  DevBuf<double> d_data_;
  std::unique_ptr<DesignCache> cache_;
  // device bases of the cache's bivariate smooths (one chunk per level batch);
  // released with the cache
  std::vector<std::unique_ptr<DevBuf<double>>> smooth_store_, smooth_spare_;

  // batch plan
  fkpc_options opt_{};
  std::vector<Test> tests_;
  std::vector<std::vector<int>> sets_;                  // unique conditioning sets
  std::vector<std::shared_ptr<const Design>> designs_;  // aligned with sets_
  std::vector<Component> comps_;
  std::vector<PairJob> pairs_;
  std::vector<FitJob> single_jobs_, multi_jobs_;
  std::vector<int> multi_small_, multi_large_, multi_huge_, multi_wide_;
  std::vector<int> direct_cols_, direct_slots_;
  // plain form: per test, offsets of its jobs in the job lists
  std::vector<int> plain_single_off_, plain_small_off_, plain_large_off_, plain_huge_off_, plain_wide_off_,
      plain_direct_off_;
  int guard_cap_ = 0;
  bool stats_enabled_ = true;

  // device buffers
  DevBuf<double> d_arena_, d_resid_, d_centre_, d_factors_, d_lr_vals_, d_lr_vecs_, d_legacy_ws_;
  DevBuf<DesignDev> d_designs_;
  DevBuf<FitJob> d_single_jobs_, d_multi_jobs_;
  DevBuf<int> d_multi_small_, d_multi_large_, d_multi_huge_, d_multi_wide_, d_direct_cols_, d_direct_slots_,
      d_comp_cols_;
  DevBuf<double> d_fit_ws_;  // global working sets of the widest fit class
  DevBuf<FitState> d_fit_states_;  // optimiser states handed to the speculative continuation
  DevBuf<int> d_defer_list_, d_defer_count_;
  // device thin-plate Lanczos of the bivariate designs
  // one set per smooth dimension (univariate, bivariate): both batches of a
  // level are in flight together
  struct TprsBuffers {
    DevBuf<double> u, V, ab, blocks, ritzp, ews, vals, zsel, U, S, colsq;
    DevBuf<int64_t> uoff, voff, roff;
    DevBuf<int> nus, done, ok, map, status;
  };
  TprsBuffers tprs_buf_[2];
  // device geometry of the additive designs
  DevBuf<GeomJob> d_geom_jobs_;
  DevBuf<WideGeomJob> d_wide_geom_jobs_;
  DevBuf<double> d_wide_log_sp_;  // kMaxPenalties log(lambda) per wide-class job
  DevBuf<SingleGeomJob> d_single_geom_jobs_;
  DevBuf<int> d_geom_status_;
  DevBuf<FitResult> d_single_res_, d_multi_res_;
  DevBuf<PairJob> d_pairs_;
  DevBuf<RecordDev> d_records_;
  DevBuf<DcovComponent> d_dcov_;
  DevBuf<HsicComponent> d_hsic_;
  DevBuf<int> d_guard_;  // [0] pair count, [1] slot count, then lists
  DevBuf<int> d_guard_mark_;  // where the late guard-band selection starts (pairs, slots)
  DevBuf<int> d_late_col_, d_part_;  // early / late split of the components and pairs
  DevBuf<DesignDev> d_designs_late_;  // descriptor array uploaded on the side stream
  bool late_designs_ = false;
  DevBuf<int> d_lr_status_;
  DevBuf<int> d_perms_;

  double* h_arena_ = nullptr;
  size_t h_arena_cap_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaEvent_t ev_[8] = {};  // [6] / [7]: the bivariate / univariate thin-plate results have landed
  std::vector<RStream>* stream_snapshots_ = nullptr;
  char* h_stage_ = nullptr;
  size_t h_stage_cap_ = 0, h_stage_used_ = 0;
  std::vector<char*> h_stage_retired_;
  // the packed descriptors, designs still pending their bivariate basis, and
  // the geometry statuses written on the device but not yet checked
  std::vector<DesignDev> ddesc_;
  std::vector<size_t> pending_;
  size_t geom_status_used_ = 0, geom_status_checked_ = 0;
  DevBuf<double> d_late_table_;
  DevBuf<SingleGeomJob> d_late_geom_jobs_;
  int launches_ = 0;
  uint64_t load_id_ = 0;
  int designs_built_ = 0;  // sets of the last batch whose design the cache lacked
  int smooths_built_ = 0;  // univariate smooths the last batch set up
  double setup_ms_ = 0.0, upload_ms_ = 0.0;
  // timeline of a one-shot batch (run_batch): host planning, host waits on
  // the device's smooth bases, and the call-start event of the device timeline
  double plan_ms_ = 0.0, smooth_wait_ms_ = 0.0, late_wait_ms_ = 0.0, tprs_host_ms_ = 0.0, design_host_ms_ = 0.0;
  bool call_timed_ = false;
  bool regress_only_ = false;  // plan_components: the targets' components only
  cudaEvent_t ev_call_ = nullptr;
  int guard_count_host_ = 0;
  double h2d_bytes_ = 0.0, d2h_bytes_ = 0.0;
  double stage_flops_[11] = {};
  bool collected_ = false;
  bool graph_timed_ = false;
  double lowrank_steps_mean_ = 0.0;
  int lowrank_steps_max_ = 0, lowrank_slots_ = 0;
  void account_flops(const std::vector<FitResult>& sres, const std::vector<FitResult>& mres);
};

}  // namespace fkpc
