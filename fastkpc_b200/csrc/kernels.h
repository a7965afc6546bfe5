// Kernel launchers (host-callable) for the fit and statistic stages.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "device.h"

namespace fkpc {

// Message for fkpc_last_error() on the calling thread.
void set_last_error(const std::string& msg);

size_t multi_smem_bytes(int qmax_class);
// Raise the dynamic shared-memory limits (call outside graph capture).
cudaError_t configure_fit_kernels();
// Raise (never lower) the statistic kernels' shared-memory limits of the
// current device to what n samples need.
cudaError_t configure_stat_kernels(int n);
// Q(a, x), the regularised upper incomplete gamma the gamma-approximation
// p-values use, for ``count`` points (ok[i] = 0: series or fraction cap hit).
cudaError_t launch_gamma_q_eval(const double* a, const double* x, int count, double* q, int* ok,
                                cudaStream_t stream);

cudaError_t launch_fit_single(const DesignDev* designs, const double* arena, const double* data, int n,
                              const FitJob* jobs, int count, double* residuals, FitResult* results,
                              cudaStream_t stream);

// Fit classes (qmax_class): 0: q <= 40, rank sum <= 32, m <= 4 (warp per fit);
// 1: q <= 76, rank sum <= 64, m <= 12; 2: q <= 112, rank sum <= 96, m <= 12
// (working set in global memory); 3: q <= 560, rank sum <= 496, m <= 62
// (working set and scalars in global memory, persistent CTAs).
// Score, gradient, Gauss-Newton and exact Hessian of GCV in log(lambda) at
// ``count`` points (rho: count x m) for design ``design`` and response y.
// qmax_class 0: q <= kWarpQ, rsum <= kWarpR, m <= kWarpM; 1: q <= 76, rsum <= 64;
// 2: q <= 112, rsum <= 96 with ``workspace`` (multi_workspace_doubles(2, count)).
cudaError_t launch_gcv_adjoint(int qmax_class, const DesignDev* designs, int design, const double* arena,
                               const double* y, int n, const double* rho, int count, double* score, double* grad,
                               double* gn, double* hess, int* status, cudaStream_t stream,
                               double* workspace = nullptr);
cudaError_t launch_fit_multi(int qmax_class, const DesignDev* designs, const double* arena, const double* data,
                             int n, const FitJob* jobs, const int* job_index, int count, double* residuals,
                             FitResult* results, cudaStream_t stream,
                             int selection = 0, double* workspace = nullptr, FitState* states = nullptr,
                             int* defer_list = nullptr, int* defer_count = nullptr,
                             cudaEvent_t after_warp = nullptr, int defer_calls = 25,
                             double* wide_log_sp = nullptr);
// (class 0: ``after_warp`` is recorded on ``stream`` once the one-warp kernel is
// queued, before the speculative continuation of the fits it deferred; class
// 3: ``wide_log_sp`` receives kMaxPenalties log(lambda) per job, in job-list
// order)
// Doubles of global workspace class ``qmax_class`` needs for ``count`` fits
// (classes 2 and 3; 0 otherwise).
size_t multi_workspace_doubles(int qmax_class, int count);

// Optional index list of a statistic launch: work item b of the grid is
// idx[b] while b < *count (both device memory), instead of b itself.  The
// grid is sized for the largest list; blocks past the count exit.
struct WorkList {
  const int* idx = nullptr;
  const int* count = nullptr;
};

// Split a level batch's components and pairs by whether their residual
// columns are final once the one-warp fit kernel has run: a column is late
// when its fit is in the speculative continuation's deferral list
// (defer_count may be NULL: nothing deferred).  With ncomp components
// (component c reads residual column c) and npairs pairs: part[0..3] =
// early / late component counts, early / late pair counts; the lists follow
// at part + 4 (early components), + ncomp (late components), + 2 ncomp
// (early pairs), + 2 ncomp + npairs (late pairs).  late_col: ncomp ints of
// scratch.  One CTA.
cudaError_t launch_stat_partition(const int* defer_list, const int* defer_count, const FitJob* jobs, int ncomp,
                                  const PairJob* pairs, int npairs, int* late_col, int* part, cudaStream_t stream);

// dCov: per component centring constants and moments, then per pair statistic
// and gamma p-value.  comp_cols[c] is the residual column of component c.
struct DcovComponent {
  double total;    // sum of distances
  double self;     // sum of squared double-centred distances
};

cudaError_t launch_dcov_components(const double* residuals, int n, const int* comp_cols, int count,
                                   double* centre, DcovComponent* comps, cudaStream_t stream, WorkList wl = {});
cudaError_t launch_dcov_pairs(const double* residuals, int n, const int* comp_cols, const double* centre,
                              const DcovComponent* comps, const PairJob* pairs, int count, RecordDev* records,
                              cudaStream_t stream, WorkList wl = {});

// Guard band: list the pairs whose exact p lies in [lo, hi] and give each of
// their components a low-rank slot.  guard layout: [0] pair count, [1] slot
// count, [2, 2+count) pair list, comp_slot[ncomp], slot_comps[cap].
// ``wl`` restricts the scan to a list of pairs.  With ``append`` the
// selection continues an earlier one (components that already hold a slot
// keep it) and first stores where it starts in mark[0] (pair list) and
// mark[1] (slots), the ``begin`` of the low-rank launches that follow it.
cudaError_t launch_guard_select(const RecordDev* records, const PairJob* pairs, int count, int ncomp, int cap,
                                double lo, double hi, int* guard, cudaStream_t stream, WorkList wl = {},
                                int append = 0, int* mark = nullptr);
// Low-rank (legacy) dCov for the guarded pairs: num_col largest-|value|
// eigenpairs per slot (vals cap x num_col, vecs n x num_col x cap, centred).
size_t legacy_eigen_workspace_doubles(int n, int ctas);
// ``slot_begin`` / ``list_begin`` (device ints, or NULL for 0): the first
// slot / guarded-pair entry this launch handles.
cudaError_t launch_legacy_eigen(const double* residuals, int n, const int* comp_cols, const int* guard,
                                const int* slot_comps, int cap, int ctas, int num_col, double* workspace,
                                double* lowrank_vals, double* lowrank_vecs, int* status, cudaStream_t stream,
                                const int* slot_begin = nullptr);
cudaError_t launch_legacy_pairs(int n, int num_col, const double* lowrank_vals, const double* lowrank_vecs,
                                const DcovComponent* comps, const int* guard, const int* guard_pairs,
                                const int* comp_slot, const PairJob* pairs, int count, RecordDev* records,
                                cudaStream_t stream, const int* list_begin = nullptr);

// HSIC: incomplete Cholesky factors (n x num_col, column-centred) per component.
struct HsicComponent {
  double offdiag;  // sum of off-diagonal entries of G G' (raw factor)
  double self;     // |Gc' Gc|_F^2
  int rank;
  int status;
};

cudaError_t launch_hsic_components(const double* residuals, int n, const int* comp_cols, int count, int num_col,
                                   double sig, double* factors, HsicComponent* comps, cudaStream_t stream,
                                   WorkList wl = {});
cudaError_t launch_hsic_pairs(int n, int num_col, const double* factors, const HsicComponent* comps,
                              const PairJob* pairs, int count, RecordDev* records, cudaStream_t stream,
                              WorkList wl = {});
cudaError_t launch_hsic_perm_pairs(int n, int num_col, const double* factors, const HsicComponent* comps,
                                   const PairJob* pairs, int count, const int* perms, int replicates,
                                   RecordDev* records, cudaStream_t stream);
cudaError_t launch_dcc_perm_pairs(const double* residuals, int n, const int* comp_cols, const double* centre,
                                  const PairJob* pairs, int count, const int* perms, int replicates,
                                  RecordDev* records, cudaStream_t stream);

// FP64 FMA throughput probe: blocks x 256 threads, 16 chains, iters steps.
cudaError_t launch_fp64_peak(double* out, int blocks, int iters, cudaStream_t stream);

// Thin-plate set-up: Lanczos on the eta matrices of a level's bivariate
// designs (one CTA per design); see kernels_tprs.cu.
constexpr int kTprsMaxSteps = 128;
constexpr int kTprsRitzMax = 30;   // Ritz pairs per design (the basis dimension k of the bivariate smooth)
constexpr int kTprsUniK = 10;      // the basis dimension k of the univariate smooth
constexpr int kTprsMaxNu = 1536;  // unique locations a design may have on the device path
// eta-matrix workspace per CTA: the leading dimension rounded up to the 32-row tile
FKPC_HD constexpr int64_t tprs_ld(int nu) { return (static_cast<int64_t>(nu) + 31) / 32 * 32; }
// Block Lanczos for bivariate designs with kTprsBlockMinNu <= nu and
// tprs_ld(nu) <= kTprsBlockMaxLd: blocks of kTprsBlock vectors, a Krylov space
// of kTprsBlockDim in kTprsBlockSteps passes over the eta matrix.
constexpr int kTprsBlock = 4;
constexpr int kTprsBlockSteps = 26;
constexpr int kTprsBlockDim = kTprsBlock * kTprsBlockSteps;
constexpr int kTprsBlockMaxLd = 512;
constexpr int kTprsBlockMinNu = kTprsBlockDim + 16;
// V: design d's nu x kTprsBlockDim basis at V + voff[d]; blocks: count x
// kTprsBlockSteps x 32 (A_s, R_s); done[d] = kTprsBlockDim, or -1 when a block
// lost a direction (the host builds that design).  ews: ctas x ews_stride.
cudaError_t launch_tprs_block_lanczos(const double* u, const int64_t* uoff, const int* nus, int count, int nu_max,
                                      double eta0, double* ews, int64_t ews_stride, int ctas, double* V,
                                      const int64_t* voff, double* blocks, int* done, cudaStream_t stream);
// Ritz pairs: vals (count x k); zsel (count x k x zstride: the selected
// eigenvectors in the Lanczos basis); ok[d] = 1 when design d's k pairs
// converged.  The select launches take the tridiagonal runs (alpha / beta /
// done of the single-vector kernel, stride steps) or the block runs; the
// vectors launch forms design d's nu x k Ritz vectors at U + uoff[d] for every
// accepted design.  k is kTprsRitzMax or kTprsUniK (block runs: kTprsRitzMax).
cudaError_t launch_tprs_ritz_select(const double* alpha, const double* beta, const int* done, int count, int steps,
                                    int k, int zstride, double* vals, double* zsel, int* ok, cudaStream_t stream);
// pws: tprs_ritz_block_workspace(count) doubles (the inner Lanczos bases).
cudaError_t launch_tprs_ritz_block_select(const double* blocks, const int* done, int count, int k, int zstride,
                                          double* pws, double* vals, double* zsel, int* ok, cudaStream_t stream);
size_t tprs_ritz_block_workspace(int count);
cudaError_t launch_tprs_ritz_vectors(const double* V, const int64_t* voff, const int* nus, const int* done,
                                     const int* ok, const double* zsel, int count, int zstride, int k, double* U,
                                     const int64_t* uoff, cudaStream_t stream);
// The thin-plate basis from its Ritz pairs (dim 2: k = kTprsRitzMax; dim 1:
// k = kTprsUniK):
// X (count x n x k doubles; design d's basis n x (k - 1) at X + d n k),
// S (count x (k-1)^2), colsq (count x (k-1)), status (count); see
// kernels_tprs.cu.
cudaError_t launch_tprs_finish(const double* U, const int64_t* uoff, const double* vals, const int* ok,
                               const double* loc, const int64_t* locoff, const int* nus, const int* mapping, int n,
                               int count, int dim, double* X, double* S, double* colsq, int* status,
                               cudaStream_t stream);
cudaError_t launch_tprs_lanczos(const double* u, const int64_t* uoff, const int* nus, int count, int nu_max, int dim,
                                int steps, double eta0, double* ews, int64_t ews_stride, int ctas, double* V,
                                const int64_t* voff, double* alpha, double* beta, int* done, cudaStream_t stream);

// Additive-design geometry (X gathered from the univariate bases, Householder
// QR, Q / R / row-packed R into the arena); see kernels_geom.cu.  status[d]:
// 1 when design d is rank deficient.  max_q <= 112 and below n.
// Single-penalty geometry (X = [1 | B], QR, whitened-penalty eigen, QW and
// spectrum into the arena); status[d] 1 rank deficient, 2 eigen failed.
cudaError_t launch_single_geometry(int n, const SingleGeomJob* jobs, int count, double* arena, int* status,
                                   cudaStream_t stream);
cudaError_t launch_additive_geometry(int n, const GeomJob* jobs, int count, int max_q, double* arena, int* status,
                                     cudaStream_t stream);
cudaError_t launch_additive_geometry(int n, const WideGeomJob* jobs, int count, int max_q, double* arena,
                                     int* status, cudaStream_t stream);

}  // namespace fkpc
