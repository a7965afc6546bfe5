// GCV smoothing-parameter selection and residuals on the GPU (FP64).
//
// fit_single_kernel: one warp per target for designs with one penalty
//   (|S| <= 2).  Spectral form of mgcv magic's GCV: with the whitened
//   penalty spectrum e_k and z = (QW)'y, the hat values are
//   h_k = 1/(1 + lambda e_k); RSS = |y|^2 - 2 sum h z^2 + sum h^2 z^2,
//   EDF = sum h, V = n RSS/(n - EDF)^2.  Newton / steepest-descent search in
//   rho = log(lambda) as in fastkpc/src/cuda/mgcv_single_penalty_gcv.cu:1479-1700
//   (15 step halvings, 400 iterations, |step| <= 5, tolerance 1e-7, boundary
//   probes of 2 up to 5 times).  Residual r = y - QW (h .* z).
//
// fit_multi_kernel: one CTA per target for additive designs (|S| > 2).
//   Each objective evaluation factors the augmented system [R; B(rho)],
//   B'B = sum_j lambda_j S_j, by Householder reflections that fold the
//   stacked penalty roots into R (shared memory, one thread per column),
//   giving Ra with Ra'Ra = X'X + S_lambda.  With W = R Ra^-1 the hat matrix is
//   Q W W' Q', so EDF = |W|_F^2 and, with g = W'Q'y,
//   RSS = |y|^2 - 2|g|^2 + |W g|^2 -- the quantities mgcv magic derives from
//   the SVD of [R; B] (fastkpc/src/mgcv_multi_penalty_cpp.cpp:732-810), in a
//   rotated basis.  The analytic gradient and Hessian in rho
//   (:834-975) use T_j = Ra^-T root_j:  M_j = T_j T_j', and every trace is a
//   small block sum over C = T'T and D = (WT)'(WT).  Newton loop of
//   :1124-1346 (25 step halvings, steepest descent after the third rejected
//   Newton trial or for an indefinite Hessian, boundary probes).
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/fastkpc_b200.h"
#include "device.h"
#include "kernels.h"

namespace fkpc {

namespace {

constexpr double kConvTol = 1e-7;
constexpr double kEps = 2.220446049250313e-16;
constexpr int kMaxIterations = 400;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// The rank rule of magic's truncated SVD (mgcv; the reference's
// rank_tolerance = sqrt(eps), fastkpc/src/cuda/mgcv_multi_penalty_gcv.hpp:230):
// an augmented pivot |Ra(c, c)| at most kRankTol times the largest one marks
// a direction in the null spaces of both X and the scaled penalties; its
// coefficient is dropped (1 / Ra(c, c) taken as 0 in every triangular solve),
// which leaves the fitted values and the influence trace of the truncated
// solution.  The fit record's flags carry kFitRankTruncated then.
constexpr double kRankTol = 1.4901161193847656e-8;
constexpr int kFitRankTruncated = kFitFlagRankTruncated;

// ----------------------------------------------------------------- single

struct SingleObjective {
  double rss, edf, score, gradient, hessian;
  bool valid;
};

__device__ double hat_value(double log_sp, double e) {
  if (e == 0.0) return 1.0;
  const double c = log_sp + log(e);
  if (c >= 0.0) {
    const double v = exp(-c);
    return v / (1.0 + v);
  }
  return 1.0 / (1.0 + exp(c));
}

// All 32 lanes call with the same log_sp; lane k < q owns component k.
// RSS = rss0 + sum_k (1 - h_k)^2 z_k^2 with rss0 = |y - QW z|^2: two sums of
// squares, so a fit that explains y almost exactly keeps a positive RSS
// (|y|^2 - 2 sum h z^2 + sum h^2 z^2 cancels to rounding noise there).
__device__ SingleObjective single_objective(double log_sp, double e, double z, bool active,
                                            double rss0, int n) {
  double lin = 0, edf = 0, rg = 0, rh = 0, dg = 0, dh = 0;
  if (active) {
    const double h = hat_value(log_sp, e);
    const double z2 = z * z;
    const double omh = 1.0 - h;
    const double w = h * omh;
    lin = omh * omh * z2;
    edf = h;
    rg = 2.0 * h * omh * omh * z2;
    rh = 2.0 * h * omh * omh * (3.0 * h - 1.0) * z2;
    dg = w;
    dh = -w * (1.0 - 2.0 * h);
  }
  lin = warp_sum(lin);
  edf = warp_sum(edf);
  rg = warp_sum(rg);
  rh = warp_sum(rh);
  dg = warp_sum(dg);
  dh = warp_sum(dh);
  SingleObjective out;
  const double rss = rss0 + lin;
  const double rdf = static_cast<double>(n) - edf;
  out.rss = rss;
  out.edf = edf;
  out.valid = isfinite(rss) && isfinite(edf) && rss > 0.0 && rdf > 1e-8;
  if (!out.valid) {
    out.score = INFINITY;
    out.gradient = NAN;
    out.hessian = NAN;
    return out;
  }
  const double score = static_cast<double>(n) * rss / (rdf * rdf);
  const double lg = rg / rss - 2.0 * dg / rdf;
  const double lh = rh / rss - (rg / rss) * (rg / rss) - 2.0 * (dh / rdf - (dg / rdf) * (dg / rdf));
  out.score = score;
  out.gradient = score * lg;
  out.hessian = score * (lh + lg * lg);
  return out;
}

}  // namespace

// The result record of one fit, written field by field (log_sp[j] for
// j < m, NaN beyond, the first kCtaPenalties), so no kernel holds a whole
// record in registers.
__device__ __forceinline__ void store_result(FitResult* __restrict__ out, const double* log_sp, int m, double score,
                                             double edf, double rss, int status, int iterations, int evaluations,
                                             int flags = 0) {
  for (int j = 0; j < kCtaPenalties; ++j) out->log_sp[j] = j < m ? log_sp[j] : NAN;
  out->score = score;
  out->edf = edf;
  out->rss = rss;
  out->status = status;
  out->iterations = iterations;
  out->evaluations = evaluations;
  out->flags = flags;
}

__global__ void fit_single_kernel(const DesignDev* __restrict__ designs, const double* __restrict__ arena,
                                  const double* __restrict__ data, int n, const FitJob* __restrict__ jobs,
                                  int job_count, double* __restrict__ residuals, FitResult* __restrict__ results) {
  const int warps = blockDim.x >> 5;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.x * warps + warp;
  if (t >= job_count) return;
  const FitJob job = jobs[t];
  const DesignDev& des = designs[job.design];
  const int q = des.q;
  const double* QW = arena + des.basis;
  const double* y = data + static_cast<int64_t>(n) * job.column;

  // z = QW' y; lane-strided rows, per-column partial sums
  double acc[kMaxSingleQ];
#pragma unroll
  for (int k = 0; k < kMaxSingleQ; ++k) acc[k] = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double yi = y[i];
#pragma unroll
    for (int k = 0; k < kMaxSingleQ; ++k)
      if (k < q) acc[k] += QW[i + static_cast<int64_t>(n) * k] * yi;
  }
  double zk = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxSingleQ; ++k) {
    const double s = warp_sum(acc[k]);
    if (k == lane) zk = s;
  }
  const bool active = lane < q;
  // rss0 = |y - QW z|^2, the part of y outside the design's span
  __shared__ double coef_all[32 * 8];
  double* coef = coef_all + warp * 32;
  coef[lane] = active ? zk : 0.0;
  __syncwarp();
  double rss0 = 0.0;
  for (int i = lane; i < n; i += 32) {
    double f = 0.0;
    for (int k = 0; k < q; ++k) f += QW[i + static_cast<int64_t>(n) * k] * coef[k];
    const double e = y[i] - f;
    rss0 += e * e;
  }
  rss0 = warp_sum(rss0);
  __syncwarp();
  const double ek = active ? arena[des.spec + lane] : 0.0;

  struct {
    int status;
  } res;
  res.status = kStatusOk;
  const int max_half = 15;
  double log_sp = des.log_sp0[0];
  SingleObjective cur = single_objective(log_sp, ek, zk, active, rss0, n);
  int calls = 1;
  int it = 0;
  bool converged = false;
  if (!cur.valid) {
    res.status = kStatusNumeric;
  } else {
    double min_score = cur.score;
    double score_red = 1e10;
    bool steepest = false;
    double prior_grad = NAN;
    double newton = 0.0, steep = 0.0;
    while (!converged && it < kMaxIterations) {
      ++it;
      bool try_step = it > 1;
      int tries = 0;
      double step = steepest ? steep : newton;
      bool src_newton = !steepest;
      bool it_flat = false;
      while (try_step) {
        ++tries;
        if (tries == 4 && !steepest) {
          steepest = true;
          step = steep;
          src_newton = false;
        }
        const double trial_ls = log_sp + step;
        const SingleObjective trial = single_objective(trial_ls, ek, zk, active, rss0, n);
        ++calls;
        const double pred = cur.gradient * step + 0.5 * cur.hessian * step * step;
        const double resolution = 8.0 * kEps * (1.0 + fabs(min_score));
        const bool unresolved = src_newton && isfinite(pred) && pred <= 0.0 && fabs(pred) <= resolution;
        if (trial.valid && trial.score < min_score) {
          try_step = false;
          score_red = min_score - trial.score;
          min_score = trial.score;
          log_sp = trial_ls;
          cur = trial;
        } else if (unresolved) {
          try_step = false;
          it_flat = true;
        } else {
          step /= 2.0;
        }
        if (tries == max_half - 1 && try_step) step = 0.0;
        if (tries == max_half) try_step = false;
      }
      if (it > 3) {
        converged = true;
        if (score_red > kConvTol * (1.0 + min_score)) converged = false;
        if (fabs(prior_grad) > pow(kConvTol, 1.0 / 3.0) * (1.0 + fabs(min_score))) converged = false;
        if (tries == max_half) converged = true;
        if (it_flat) converged = true;
      }
      prior_grad = cur.gradient;
      steepest = cur.hessian < 0.0;
      if (!steepest) {
        newton = -cur.gradient / cur.hessian;
        if (fabs(newton) > 5.0) newton = copysign(5.0, newton);
      }
      steep = cur.gradient == 0.0 ? 0.0 : -cur.gradient / fabs(cur.gradient);
    }
    if (!converged) {
      res.status = kStatusNotConverged;
    } else {
      const double direction = cur.gradient < 0.0 ? 1.0 : -1.0;
      for (int probe = 0; probe < 5; ++probe) {
        const double trial_ls = log_sp + direction * 2.0;
        const SingleObjective trial = single_objective(trial_ls, ek, zk, active, rss0, n);
        ++calls;
        if (!(trial.valid && trial.score < min_score)) break;
        log_sp = trial_ls;
        cur = trial;
        min_score = trial.score;
      }
      // terminal Newton polish to the stationary point: magic's stopping rule
      // fixes rho only to about its tolerance, a few Newton steps (taken only
      // when small, with positive curvature) make the selected point
      // reproducible to rounding
      for (int ps = 0; ps < 4; ++ps) {
        if (!(cur.valid && cur.hessian > 1e-6 * cur.score)) break;
        const double step = -cur.gradient / cur.hessian;
        if (fabs(step) > 1e-6) break;
        log_sp += step;
        cur = single_objective(log_sp, ek, zk, active, rss0, n);
        ++calls;
        if (fabs(step) <= 1e-10) break;
      }
    }
  }
  // residual r = y - QW (h .* z)
  coef[lane] = active ? hat_value(log_sp, ek) * zk : 0.0;
  __syncwarp();
  double* r = residuals + static_cast<int64_t>(n) * job.out;
  for (int i = lane; i < n; i += 32) {
    double f = 0.0;
    for (int k = 0; k < q; ++k) f += QW[i + static_cast<int64_t>(n) * k] * coef[k];
    r[i] = y[i] - f;
  }
  if (lane == 0) store_result(results + t, &log_sp, 1, cur.score, cur.edf, cur.rss, res.status, it, calls);
}

// ----------------------------------------------------------------- multi

namespace {

constexpr int kMultiThreads = 128;
constexpr int kPolishSteps = 4;
constexpr double kPolishMaxStep = 1e-6;
constexpr double kPolishDone = 1e-10;
constexpr double kPolishCurvature = 1e-6;
constexpr double kGnGradTol = 1e-9;   // Gauss-Newton selection: |grad V| <= 1e-9 (1 + V),
constexpr double kGnFlatTol = 1e-12;  // or a decrease <= 1e-12 (1 + V)
constexpr double kGnFlatGrad = 1e-6;  // with |grad V| <= 1e-6 (1 + V),
constexpr double kGnStallTol = 1e-9;   // a decrease of V at most 1e-9 (1 + V): the direction has stalled
constexpr double kGnMaxLogSp = 25.0;  // upper bound of the Gauss-Newton search in log(lambda)

__device__ __forceinline__ int tri(int i, int j) { return j * (j + 1) / 2 + i; }  // packed upper, i <= j

template <int QMAX, int RMAX>
struct MultiLayout {
  static constexpr int TRI = QMAX * (QMAX + 1) / 2;
  static constexpr int LDB = RMAX + 1;  // odd leading dimensions: conflict-free column walks
  static constexpr int LDT = QMAX + 1;
  static constexpr int BSZ = (LDB * QMAX > LDT * RMAX) ? LDB * QMAX : LDT * RMAX;
  static constexpr int RS = 0;         // R of the design, packed upper (staged once per target)
  static constexpr int RA = RS + TRI;
  static constexpr int W = RA + TRI;
  static constexpr int B = W + TRI;  // stacked penalty roots, then T = Ra^-T root
  static constexpr int WT = B + BSZ;
  static constexpr int Y0 = WT + LDT * RMAX;
  static constexpr int G = Y0 + QMAX;
  static constexpr int WG = G + QMAX;
  static constexpr int E1 = WG + QMAX;
  static constexpr int AV = E1 + QMAX;
  static constexpr int BV = AV + RMAX;
  static constexpr int IDG = BV + RMAX;  // 1 / Ra(c, c)
  static constexpr int TOTAL = IDG + QMAX;
};

// Scalars and index maps of one CTA-class fit: at most MP penalties, NT
// threads, QC coefficients and RC stacked root rows.
template <int MP, int NT, int QC, int RC>
struct MultiScalarsT {
  static constexpr int kLd = MP;  // leading dimension of the m x m matrices
  static constexpr int kThreads = NT;
  double beta[2], v0[2];
  double red[NT / 32];
  double score, rss, edf, rss0;  // rss0 = |y - Q Q'y|^2
  int dropped;                   // coefficients the rank rule dropped at the last evaluation
  double lam[MP];
  double log_sp[MP];
  double trial[MP];
  double step[MP];
  double grad_c[MP];
  double hess_c[MP * MP];
  double gn_c[MP * MP];  // Gauss-Newton Hessian (adjoint entry point)
  double gradient[MP];
  double newton[MP];
  double steep[MP];
  double ddelta[MP];
  double drss[MP];
  int status;
  int nzrow[QC];
  int col_block[RC];
  int pair_i[MP * (MP + 1) / 2];
  int pair_j[MP * (MP + 1) / 2];
  double ja[MP * MP];  // thread-0 scratch: Jacobi matrix / Cholesky factor
  double jv[MP * MP];  // Jacobi rotations
};
// the shared-memory classes (q <= 112, |S| <= 12)
using MultiScalars = MultiScalarsT<kCtaPenalties, kMultiThreads, 128, 128>;

template <class S>
__device__ double block_max(double v, S* sc) {
  v = warp_max(v);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sc->red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < S::kThreads / 32; ++w) s = fmax(s, sc->red[w]);
  return s;
}

template <class S>
__device__ double block_sum(double v, S* sc) {
  v = warp_sum(v);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sc->red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < S::kThreads / 32; ++w) s += sc->red[w];
  return s;
}

// Objective at sc->trial: fold the stacked roots into R (Ra'Ra = X'X + S),
// W = R Ra^-1 by row solves, g = W'y0, W g, EDF, RSS, score.  Leaves Ra, W,
// g, Wg in shared memory for multi_derivatives.
template <int QMAX, int RMAX, class S = MultiScalars, class D = DesignDev>
__device__ void multi_core(const D& des, const double* __restrict__ arena, int n, double* sm, S* sc) {
  using L = MultiLayout<QMAX, RMAX>;
  constexpr int NT = S::kThreads;
  const int tid = threadIdx.x;
  const int q = des.q, m = des.m;
  double* Ra = sm + L::RA;
  double* W = sm + L::W;
  double* B = sm + L::B;
  const double* Rs = sm + L::RS;
  double* idg = sm + L::IDG;
  const double* roots = arena + des.roots;
  for (int j = tid; j < m; j += NT) sc->lam[j] = exp(sc->trial[j]);
  for (int idx = tid; idx < L::LDB * q; idx += NT) B[idx] = 0.0;
  for (int idx = tid; idx < q * (q + 1) / 2; idx += NT) Ra[idx] = Rs[idx];
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    const double s = sqrt(sc->lam[j]);
    const int dim = des.dim[j], rk = des.rank[j];
    const double* root = roots + des.rootoff[j];
    for (int idx = tid; idx < dim * rk; idx += NT) {
      const int a = idx % dim, c = idx / dim;  // root[a + dim c] -> B[rowoff + c, off + a]
      B[(des.rowoff[j] + c) + L::LDB * (des.off[j] + a)] = s * root[idx];
    }
  }
  __syncthreads();
  for (int k = 0; k < q; ++k) {
    // reflector for column k: warp 0 reduces |B[0..nz, k]|^2
    const int nz = sc->nzrow[k];
    const double* Bk = B + L::LDB * k;
    if (tid < 32) {
      double sg = 0.0;
      for (int i = tid; i < nz; i += 32) sg += Bk[i] * Bk[i];
      sg = warp_sum(sg);
      if (tid == 0) {
        const double akk = Ra[tri(k, k)];
        if (sg == 0.0) {
          sc->beta[0] = 0.0;
          sc->v0[0] = 0.0;
        } else {
          const double nrm = sqrt(akk * akk + sg);
          const double alpha = akk >= 0.0 ? -nrm : nrm;
          const double v0 = akk - alpha;
          sc->beta[0] = 2.0 / (v0 * v0 + sg);
          sc->v0[0] = v0;
          Ra[tri(k, k)] = alpha;
        }
      }
    }
    __syncthreads();
    const double beta = sc->beta[0];
    const double v0 = sc->v0[0];
    for (int j = k + 1 + tid; beta != 0.0 && j < q; j += NT) {
      double* Bj = B + L::LDB * j;
      double w0 = v0 * Ra[tri(k, j)], w1 = 0.0, w2 = 0.0, w3 = 0.0;
      int i = 0;
      for (; i + 3 < nz; i += 4) {
        w0 += Bk[i] * Bj[i];
        w1 += Bk[i + 1] * Bj[i + 1];
        w2 += Bk[i + 2] * Bj[i + 2];
        w3 += Bk[i + 3] * Bj[i + 3];
      }
      for (; i < nz; ++i) w0 += Bk[i] * Bj[i];
      const double w = beta * ((w0 + w1) + (w2 + w3));
      Ra[tri(k, j)] -= w * v0;
      for (int r = 0; r < nz; ++r) Bj[r] -= w * Bk[r];
    }
    __syncthreads();
  }
  // reciprocal diagonal once, so the triangular solves below multiply; the
  // rank rule drops the coefficients of negligible pivots
  double dmax = 0.0;
  for (int c = tid; c < q; c += NT) dmax = fmax(dmax, fabs(Ra[tri(c, c)]));
  dmax = block_max(dmax, sc);
  double dropped = 0.0;
  for (int c = tid; c < q; c += NT) {
    const double dc = Ra[tri(c, c)];
    const bool keep = fabs(dc) > kRankTol * dmax;
    idg[c] = keep ? 1.0 / dc : 0.0;
    dropped += keep ? 0.0 : 1.0;
  }
  dropped = block_sum(dropped, sc);
  if (tid == 0) {
    sc->dropped = static_cast<int>(dropped);
    if (!(dmax > 0.0)) sc->status = kStatusRank;
  }
  __syncthreads();
  // W = R Ra^-1: row i solves w Ra = R(i, :), w upper triangular
  for (int i = tid; i < q; i += NT) {
    for (int c = i; c < q; ++c) {
      const double* rac = Ra + c * (c + 1) / 2;  // column c of Ra
      double s0 = Rs[tri(i, c)], s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int t = i;
      for (; t + 3 < c; t += 4) {
        s0 -= W[tri(i, t)] * rac[t];
        s1 -= W[tri(i, t + 1)] * rac[t + 1];
        s2 -= W[tri(i, t + 2)] * rac[t + 2];
        s3 -= W[tri(i, t + 3)] * rac[t + 3];
      }
      for (; t < c; ++t) s0 -= W[tri(i, t)] * rac[t];
      W[tri(i, c)] = ((s0 + s1) + (s2 + s3)) * idg[c];
    }
  }
  __syncthreads();
  double* y0 = sm + L::Y0;
  double* g = sm + L::G;
  double* Wg = sm + L::WG;
  double e = 0.0;
  for (int c = tid; c < q; c += NT) {
    double s = 0.0;
    for (int i = 0; i <= c; ++i) {
      const double w = W[tri(i, c)];
      s += w * y0[i];
      e += w * w;
    }
    g[c] = s;
  }
  const double edf = block_sum(e, sc);
  // RSS = |y - Q y0|^2 + |y0 - W g|^2: sums of squares, no cancellation
  double gg = 0.0;
  for (int i = tid; i < q; i += NT) {
    double s = 0.0;
    for (int c = i; c < q; ++c) s += W[tri(i, c)] * g[c];
    Wg[i] = s;
    const double d = y0[i] - s;
    gg += d * d;
  }
  const double part = block_sum(gg, sc);
  if (tid == 0) {
    const double rss = sc->rss0 + part;
    const double delta = static_cast<double>(n) - edf;
    sc->rss = rss;
    sc->edf = edf;
    if (!(isfinite(rss) && isfinite(edf)) || delta <= 1e-8) {
      sc->score = INFINITY;
      if (sc->status == kStatusOk) sc->status = kStatusNumeric;
    } else {
      sc->score = static_cast<double>(n) * rss / (delta * delta);
    }
  }
  __syncthreads();
}

// Gradient and Hessian of V at the point of the last multi_core call.
// M_j = T_j T_j' with T = Ra^-T root; with C = T'T and D = (WT)'(WT) every
// trace is a block sum: d delta_j = lam_j sum_{a in j} D_aa,
// d rss_j = 2 lam_j b_j'a_j, tr(M_i M_j P) = sum C_ab D_ab over block (i, j).
template <int QMAX, int RMAX, class S = MultiScalars, class D = DesignDev>
__device__ void multi_derivatives(const D& des, const double* __restrict__ arena, int n, double* sm, S* sc) {
  using L = MultiLayout<QMAX, RMAX>;
  constexpr int NT = S::kThreads;
  const int tid = threadIdx.x;
  const int q = des.q, m = des.m, rs = des.rsum;
  const double* Ra = sm + L::RA;
  const double* W = sm + L::W;
  double* T = sm + L::B;
  double* WT = sm + L::WT;
  const double* g = sm + L::G;
  const double* Wg = sm + L::WG;
  double* e1 = sm + L::E1;
  double* av = sm + L::AV;
  double* bv = sm + L::BV;
  const double* roots = arena + des.roots;
  // T(:, col) = Ra^-T root(:, col): forward substitution, one thread per column
  for (int col = tid; col < rs; col += NT) {
    const int j = sc->col_block[col];
    const int c = col - des.rowoff[j];
    const int off = des.off[j], dim = des.dim[j];
    const double* root = roots + des.rootoff[j];
    for (int i = 0; i < off; ++i) T[i + L::LDT * col] = 0.0;
    const double* idg = sm + L::IDG;
    double* Tc = T + L::LDT * col;
    for (int i = off; i < q; ++i) {
      const double* rai = Ra + i * (i + 1) / 2;  // column i of Ra
      double s0 = (i < off + dim) ? root[(i - off) + dim * c] : 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int t = off;
      for (; t + 3 < i; t += 4) {
        s0 -= rai[t] * Tc[t];
        s1 -= rai[t + 1] * Tc[t + 1];
        s2 -= rai[t + 2] * Tc[t + 2];
        s3 -= rai[t + 3] * Tc[t + 3];
      }
      for (; t < i; ++t) s0 -= rai[t] * Tc[t];
      Tc[i] = ((s0 + s1) + (s2 + s3)) * idg[i];
    }
  }
  // e1 = g - W'(W g)
  for (int c = tid; c < q; c += NT) {
    double s = 0.0;
    for (int i = 0; i <= c; ++i) s += W[tri(i, c)] * Wg[i];
    e1[c] = g[c] - s;
  }
  __syncthreads();
  // W T, a = T'g, b = T'e1
  for (int idx = tid; idx < q * rs; idx += NT) {
    const int i = idx % q, col = idx / q;
    const int j = sc->col_block[col];
    double s = 0.0;
    for (int t = max(i, des.off[j]); t < q; ++t) s += W[tri(i, t)] * T[t + L::LDT * col];
    WT[i + L::LDT * col] = s;
  }
  for (int col = tid; col < rs; col += NT) {
    double sa = 0.0, sb = 0.0;
    for (int i = 0; i < q; ++i) {
      const double tv = T[i + L::LDT * col];
      sa += tv * g[i];
      sb += tv * e1[i];
    }
    av[col] = sa;
    bv[col] = sb;
  }
  __syncthreads();
  for (int j = tid; j < m; j += NT) {
    double dd = 0.0, dr = 0.0;
    for (int a = des.rowoff[j]; a < des.rowoff[j] + des.rank[j]; ++a) {
      double d = 0.0;
      for (int i = 0; i < q; ++i) d += WT[i + L::LDT * a] * WT[i + L::LDT * a];
      dd += d;
      dr += bv[a] * av[a];
    }
    sc->ddelta[j] = sc->lam[j] * dd;
    sc->drss[j] = 2.0 * sc->lam[j] * dr;
  }
  __syncthreads();
  const double nd = static_cast<double>(n);
  const double delta = nd - sc->edf;
  const double s1 = nd / (delta * delta);
  const double s2 = 2.0 * s1 * sc->rss / delta;
  const int npair = m * (m + 1) / 2;
  const int warp = tid >> 5, lane = tid & 31;
  for (int pidx = warp; pidx < npair; pidx += NT / 32) {
    const int bi = sc->pair_i[pidx], bj = sc->pair_j[pidx];
    const int ri = des.rank[bi], rj = des.rank[bj];
    const int oi = des.rowoff[bi], oj = des.rowoff[bj];
    double trmmp = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (int e = lane; e < ri * rj; e += 32) {
      const int a = oi + e % ri, b = oj + e / ri;
      double cab = 0.0, dab = 0.0;
      for (int i = 0; i < q; ++i) {
        cab += T[i + L::LDT * a] * T[i + L::LDT * b];
        dab += WT[i + L::LDT * a] * WT[i + L::LDT * b];
      }
      trmmp += cab * dab;
      t1 += av[b] * dab * av[a];  // a_j' D_ji a_i
      t2 += bv[a] * cab * av[b];  // b_i' C_ij a_j
      t3 += bv[b] * cab * av[a];  // b_j' C_ji a_i
    }
    trmmp = warp_sum(trmmp);
    t1 = warp_sum(t1);
    t2 = warp_sum(t2);
    t3 = warp_sum(t3);
    if (lane == 0) {
      const double ll = sc->lam[bi] * sc->lam[bj];
      double d2delta = -2.0 * ll * trmmp;
      double d2rss = 2.0 * ll * (t1 - t2 - t3);
      if (bi == bj) {
        d2delta += sc->ddelta[bi];
        d2rss += sc->drss[bi];
      }
      const double h = -2.0 * s1 / delta * (sc->ddelta[bj] * sc->drss[bi] + sc->ddelta[bi] * sc->drss[bj]) +
                       s1 * d2rss + 3.0 * s2 / delta * sc->ddelta[bi] * sc->ddelta[bj] - s2 * d2delta;
      sc->hess_c[bi + S::kLd * bj] = h;
      sc->hess_c[bj + S::kLd * bi] = h;
      // Gauss-Newton: V = |f|^2, f = sqrt(n) r / delta, dr_i . dr_j = ll a_i' D_ij a_j
      const double gn = 2.0 * s1 * ll * t1 - s1 / delta * (sc->ddelta[bj] * sc->drss[bi] + sc->ddelta[bi] * sc->drss[bj]) +
                        s2 / delta * sc->ddelta[bi] * sc->ddelta[bj];
      sc->gn_c[bi + S::kLd * bj] = gn;
      sc->gn_c[bj + S::kLd * bi] = gn;
    }
  }
  for (int j = tid; j < m; j += NT) sc->grad_c[j] = s1 * sc->drss[j] - s2 * sc->ddelta[j];
  __syncthreads();
}

// Newton step from the Hessian eigen-decomposition (cyclic Jacobi, m <= 8).
template <class S>
__device__ void newton_from_hessian_eigen(int m, S* sc, bool* steepest) {
  double* a = sc->ja;
  double* v = sc->jv;
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      a[i + S::kLd * j] = sc->hess_c[i + S::kLd * j];
      v[i + S::kLd * j] = i == j ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) {
        const double x = a[i + S::kLd * j];
        if (i == j) dg += x * x;
        else off += x * x;
      }
    if (off == 0.0 || off <= 1e-32 * dg) break;
    for (int p = 0; p < m - 1; ++p)
      for (int r = p + 1; r < m; ++r) {
        const double apq = a[p + S::kLd * r];
        if (apq == 0.0) continue;
        const double theta = (a[r + S::kLd * r] - a[p + S::kLd * p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        for (int k = 0; k < m; ++k) {
          const double akp = a[k + S::kLd * p], akq = a[k + S::kLd * r];
          a[k + S::kLd * p] = c * akp - s * akq;
          a[k + S::kLd * r] = s * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {
          const double apk = a[p + S::kLd * k], aqk = a[r + S::kLd * k];
          a[p + S::kLd * k] = c * apk - s * aqk;
          a[r + S::kLd * k] = s * apk + c * aqk;
        }
        a[p + S::kLd * r] = 0.0;
        a[r + S::kLd * p] = 0.0;
        for (int k = 0; k < m; ++k) {
          const double vkp = v[k + S::kLd * p], vkq = v[k + S::kLd * r];
          v[k + S::kLd * p] = c * vkp - s * vkq;
          v[k + S::kLd * r] = s * vkp + c * vkq;
        }
      }
  }
  bool neg = false;
  for (int j = 0; j < m; ++j)
    if (a[j + S::kLd * j] < 0.0) neg = true;
  *steepest = neg;
  if (!neg) {
    double proj[S::kLd];
    for (int c = 0; c < m; ++c) {
      double s = 0.0;
      for (int r = 0; r < m; ++r) s += v[r + S::kLd * c] * sc->gradient[r];
      proj[c] = s / a[c + S::kLd * c];
    }
    double mx = 0.0;
    for (int r = 0; r < m; ++r) {
      double s = 0.0;
      for (int c = 0; c < m; ++c) s += v[r + S::kLd * c] * proj[c];
      sc->newton[r] = -s;
      mx = fmax(mx, fabs(sc->newton[r]));
    }
    if (mx > 5.0)
      for (int r = 0; r < m; ++r) sc->newton[r] *= 5.0 / mx;
  }
  double mg = 0.0;
  for (int r = 0; r < m; ++r) mg = fmax(mg, fabs(sc->gradient[r]));
  for (int r = 0; r < m; ++r) sc->steep[r] = mg == 0.0 ? 0.0 : -sc->gradient[r] / mg;
}

// Newton step for the magic loop (one thread).  A positive definite Hessian
// (Cholesky succeeds) gives the Newton step -H^-1 g from the factor; when
// Cholesky fails the eigen-decomposition decides, as in the reference: any
// negative eigenvalue selects steepest descent.  The step is capped at 5 in
// max norm and the steepest-descent direction is -g / max|g|.
template <class S>
__device__ void newton_from_hessian(int m, S* sc, bool* steepest) {
  double* Lm = sc->ja;
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < m; ++r) Lm[r + S::kLd * c] = sc->hess_c[r + S::kLd * c];
  bool pd = true;
  for (int c = 0; c < m && pd; ++c) {
    double d = Lm[c + S::kLd * c];
    for (int k = 0; k < c; ++k) d -= Lm[c + S::kLd * k] * Lm[c + S::kLd * k];
    if (!(d > 0.0)) {
      pd = false;
      break;
    }
    d = sqrt(d);
    Lm[c + S::kLd * c] = d;
    const double inv = 1.0 / d;
    for (int r = c + 1; r < m; ++r) {
      double s = Lm[r + S::kLd * c];
      for (int k = 0; k < c; ++k) s -= Lm[r + S::kLd * k] * Lm[c + S::kLd * k];
      Lm[r + S::kLd * c] = s * inv;
    }
  }
  if (!pd) {
    newton_from_hessian_eigen(m, sc, steepest);
    return;
  }
  *steepest = false;
  double z[S::kLd];
  for (int r = 0; r < m; ++r) {
    double s = -sc->gradient[r];
    for (int k = 0; k < r; ++k) s -= Lm[r + S::kLd * k] * z[k];
    z[r] = s / Lm[r + S::kLd * r];
  }
  double mx = 0.0;
  for (int r = m - 1; r >= 0; --r) {
    double s = z[r];
    for (int k = r + 1; k < m; ++k) s -= Lm[k + S::kLd * r] * z[k];
    z[r] = s / Lm[r + S::kLd * r];
    mx = fmax(mx, fabs(z[r]));
  }
  for (int r = 0; r < m; ++r) sc->newton[r] = mx > 5.0 ? z[r] * (5.0 / mx) : z[r];
  double mg = 0.0;
  for (int r = 0; r < m; ++r) mg = fmax(mg, fabs(sc->gradient[r]));
  for (int r = 0; r < m; ++r) sc->steep[r] = mg == 0.0 ? 0.0 : -sc->gradient[r] / mg;
}

// Terminal Newton polish (one thread): Newton step on the coordinates whose
// curvature exceeds kPolishCurvature * V, by Cholesky of that sub-Hessian.
// Returns 0 to stop (no active coordinate, indefinite, or step too large),
// 1 when the step was applied, 2 when it was applied and was negligible.
template <class S>
__device__ int polish_step(int m, S* sc) {
  int act[S::kLd];
  int na = 0;
  for (int j = 0; j < m; ++j)
    if (sc->hess_c[j + S::kLd * j] > kPolishCurvature * sc->score) act[na++] = j;
  if (na == 0) return 0;
  double* Lm = sc->ja;
  for (int c = 0; c < na; ++c)
    for (int r = 0; r < na; ++r) Lm[r + S::kLd * c] = sc->hess_c[act[r] + S::kLd * act[c]];
  for (int c = 0; c < na; ++c) {
    double d = Lm[c + S::kLd * c];
    for (int k = 0; k < c; ++k) d -= Lm[c + S::kLd * k] * Lm[c + S::kLd * k];
    if (!(d > 0.0)) return 0;
    d = sqrt(d);
    Lm[c + S::kLd * c] = d;
    for (int r = c + 1; r < na; ++r) {
      double s = Lm[r + S::kLd * c];
      for (int k = 0; k < c; ++k) s -= Lm[r + S::kLd * k] * Lm[c + S::kLd * k];
      Lm[r + S::kLd * c] = s / d;
    }
  }
  double z[S::kLd];
  for (int r = 0; r < na; ++r) {
    double s = -sc->grad_c[act[r]];
    for (int k = 0; k < r; ++k) s -= Lm[r + S::kLd * k] * z[k];
    z[r] = s / Lm[r + S::kLd * r];
  }
  double mx = 0.0;
  for (int r = na - 1; r >= 0; --r) {
    double s = z[r];
    for (int k = r + 1; k < na; ++k) s -= Lm[k + S::kLd * r] * z[k];
    z[r] = s / Lm[r + S::kLd * r];
    mx = fmax(mx, fabs(z[r]));
  }
  if (mx > kPolishMaxStep) return 0;
  for (int r = 0; r < na; ++r) sc->log_sp[act[r]] += z[r];
  return mx <= kPolishDone ? 2 : 1;
}

// Cholesky solve of (A + mu I) z = -g (one thread, m <= 62, A column-major
// with leading dimension ld) on the coordinates whose bit in ``fixed`` is
// clear; fixed coordinates get z = 0.  False when the factor does not exist.
__device__ bool chol_solve_neg(int m, int ld, const double* A, double mu, const double* g,
                               unsigned long long fixed, double* Lm, double* z) {
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < m; ++r) {
      const bool fr = (fixed >> r) & 1ull, fc = (fixed >> c) & 1ull;
      Lm[r + ld * c] = (fr || fc) ? (r == c ? 1.0 : 0.0) : A[r + ld * c] + (r == c ? mu : 0.0);
    }
  for (int c = 0; c < m; ++c) {
    double d = Lm[c + ld * c];
    for (int k = 0; k < c; ++k) d -= Lm[c + ld * k] * Lm[c + ld * k];
    if (!(d > 0.0)) return false;
    d = sqrt(d);
    Lm[c + ld * c] = d;
    for (int r = c + 1; r < m; ++r) {
      double v = Lm[r + ld * c];
      for (int k = 0; k < c; ++k) v -= Lm[r + ld * k] * Lm[c + ld * k];
      Lm[r + ld * c] = v / d;
    }
  }
  for (int r = 0; r < m; ++r) {
    double v = ((fixed >> r) & 1ull) ? 0.0 : -g[r];
    for (int k = 0; k < r; ++k) v -= Lm[r + ld * k] * z[k];
    z[r] = v / Lm[r + ld * r];
  }
  for (int r = m - 1; r >= 0; --r) {
    double v = z[r];
    for (int k = r + 1; k < m; ++k) v -= Lm[k + ld * r] * z[k];
    z[r] = v / Lm[r + ld * r];
  }
  return true;
}

// Newton or damped Gauss-Newton solve of the adjoint-driven selection on the
// free coordinates (see gn_step).  False when no factor exists.
template <class S>
__device__ bool gn_solve(int m, S* sc, unsigned long long fixed, double* z) {
  if (chol_solve_neg(m, S::kLd, sc->hess_c, 0.0, sc->grad_c, fixed, sc->ja, z)) return true;
  double dmax = 0.0;
  for (int j = 0; j < m; ++j) dmax = fmax(dmax, fabs(sc->gn_c[j + S::kLd * j]));
  double mu = 0.0;
  for (int attempt = 0; attempt < 12; ++attempt) {
    if (chol_solve_neg(m, S::kLd, sc->gn_c, mu, sc->grad_c, fixed, sc->ja, z)) return true;
    mu = mu == 0.0 ? 1e-12 * fmax(dmax, 1e-300) : mu * 100.0;
  }
  return false;
}

// Step of the adjoint-driven selection (one thread): Newton on the exact
// Hessian where it is positive definite (quadratic convergence near a
// minimum), else on the Gauss-Newton Hessian GN = 2 J'J (positive
// semi-definite, singular in the flat directions of V) damped by mu = 1e-12,
// 1e-10, ... times its largest diagonal entry until Cholesky succeeds.
// Projected on the bound log(lambda) <= kGnMaxLogSp: coordinates on the
// bound whose step points outwards are fixed and the rest re-solved.  The
// step is capped at 5 in max norm as magic's.
template <class S>
__device__ void gn_step(int m, S* sc) {
  double z[S::kLd];
  unsigned long long fixed = 0ull;
  bool ok = gn_solve(m, sc, fixed, z);
  if (ok) {
    for (int r = 0; r < m; ++r)
      if (sc->log_sp[r] >= kGnMaxLogSp && z[r] > 0.0) fixed |= 1ull << r;
    if (fixed) ok = gn_solve(m, sc, fixed, z);
  }
  if (!ok) {
    double mg = 0.0;
    for (int r = 0; r < m; ++r) mg = fmax(mg, fabs(sc->grad_c[r]));
    for (int r = 0; r < m; ++r) z[r] = mg == 0.0 ? 0.0 : -sc->grad_c[r] / mg;
  }
  double mx = 0.0;
  for (int r = 0; r < m; ++r) mx = fmax(mx, fabs(z[r]));
  for (int r = 0; r < m; ++r) {
    const double st = mx > 5.0 ? z[r] * (5.0 / mx) : z[r];
    // the unpivoted fold loses accuracy in the penalty null spaces as
    // log(lambda) grows (about 1e-16 sqrt(lambda) relative), and V is flat
    // there: the search stays below kGnMaxLogSp
    sc->step[r] = fmin(st, kGnMaxLogSp - sc->log_sp[r]);
  }
}

// Projected steepest descent for a stalled Gauss-Newton search (one
// thread): -g / max|g| over the coordinates that no outward push holds at
// the bound log(lambda) <= kGnMaxLogSp, clipped to the bound.
template <class S>
__device__ void gn_steepest(int m, S* sc) {
  double mg = 0.0;
  for (int r = 0; r < m; ++r)
    if (!(sc->log_sp[r] >= kGnMaxLogSp && sc->gradient[r] < 0.0)) mg = fmax(mg, fabs(sc->gradient[r]));
  for (int r = 0; r < m; ++r) {
    const bool held = sc->log_sp[r] >= kGnMaxLogSp && sc->gradient[r] < 0.0;
    const double z = (mg == 0.0 || held) ? 0.0 : -sc->gradient[r] / mg;
    sc->step[r] = fmin(z, kGnMaxLogSp - sc->log_sp[r]);
  }
}

}  // namespace

// Per-fit set-up shared by the fit and adjoint kernels: fill-in bounds, block
// maps, R staged in shared memory, y0 = Q'y and |y|^2.
template <int QMAX, int RMAX, class S = MultiScalars, class D = DesignDev>
__device__ void multi_fit_setup(const D& des, const double* __restrict__ arena, const double* __restrict__ y,
                                int n, double* sm, S& sc) {
  using L = MultiLayout<QMAX, RMAX>;
  constexpr int NT = S::kThreads;
  const int tid = threadIdx.x;
  const int q = des.q, m = des.m;
  const double* Q = arena + des.basis;
  if (tid == 0) {
    sc.status = kStatusOk;
    int row = 0;
    for (int c = 0; c < q; ++c) {
      int nz = 0;
      for (int j = 0; j < m; ++j)
        if (des.off[j] <= c) nz = des.rowoff[j] + des.rank[j];
      sc.nzrow[c] = nz;
    }
    for (int j = 0; j < m; ++j)
      for (int c = 0; c < des.rank[j]; ++c) sc.col_block[row++] = j;
    int pp = 0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j <= i; ++j) {
        sc.pair_i[pp] = i;
        sc.pair_j[pp] = j;
        ++pp;
      }
  }
  {
    const double* R = arena + des.rmat;
    double* Rs = sm + L::RS;
    for (int c = 0; c < q; ++c)
      for (int i = tid; i <= c; i += NT) Rs[tri(i, c)] = R[i + static_cast<int64_t>(q) * c];
  }
  // y0 = Q'y and rss0 = |y - Q y0|^2
  double* y0 = sm + L::Y0;
  {
    const int warp = tid >> 5, lane = tid & 31;
    for (int c = warp; c < q; c += NT / 32) {
      double s = 0.0;
      for (int i = lane; i < n; i += 32) s += Q[i + static_cast<int64_t>(n) * c] * y[i];
      s = warp_sum(s);
      if (lane == 0) y0[c] = s;
    }
    __syncthreads();
    double ee = 0.0;
    for (int i = tid; i < n; i += NT) {
      double f = 0.0;
      for (int c = 0; c < q; ++c) f += Q[i + static_cast<int64_t>(n) * c] * y0[c];
      const double e = y[i] - f;
      ee += e * e;
    }
    ee = block_sum(ee, &sc);
    if (tid == 0) sc.rss0 = ee;
  }
}

// One fit of a CTA class: magic's search (or the Gauss-Newton selection),
// boundary probes, polish, residual and result record.  sm: the working set
// (shared or global), sc: the scalars, ctl: 4 shared ints.
template <int QMAX, int RMAX, class S, class D>
__device__ void multi_fit_job(const D& des, const FitJob& job, int t, const double* __restrict__ arena,
                              const double* __restrict__ data, int n, double* __restrict__ residuals,
                              FitResult* __restrict__ results, int selection, double* sm, S& sc, int* ctl,
                              double* __restrict__ all_log_sp) {
  using L = MultiLayout<QMAX, RMAX>;
  constexpr int NT = S::kThreads;
  const int tid = threadIdx.x;
  const int q = des.q, m = des.m;
  const double* y = data + static_cast<int64_t>(n) * job.column;
  const double* Q = arena + des.basis;
  multi_fit_setup<QMAX, RMAX, S, D>(des, arena, y, n, sm, sc);
  if (tid < m) {
    sc.log_sp[tid] = des.log_sp0[tid];
    sc.trial[tid] = des.log_sp0[tid];
  }
  __syncthreads();
  multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
  multi_derivatives<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
  double min_score = sc.score;
  double score_red = 1e10;
  bool steepest = false;
  bool converged = false;
  int calls = 1;
  int it = 0;
  const int max_half = 25;
  if (tid < m) {
    sc.gradient[tid] = 0.0;
    sc.newton[tid] = 0.0;
    sc.steep[tid] = 0.0;
  }
  __syncthreads();
  if (selection == FKPC_SELECT_GN_NEWTON) {
    // Newton on the Gauss-Newton Hessian, halving until V decreases
    if (tid < m) sc.gradient[tid] = sc.grad_c[tid];
    __syncthreads();
    bool stalled = false;
    for (it = 1; it <= kMaxIterations && sc.status == kStatusOk; ++it) {
      if (tid == 0) {
        if (stalled) gn_steepest(m, &sc);
        else gn_step(m, &sc);
      }
      __syncthreads();
      bool accepted = false;
      for (int tries = 1; tries <= max_half; ++tries) {
        if (tid < m) sc.trial[tid] = sc.log_sp[tid] + sc.step[tid];
        __syncthreads();
        multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
        ++calls;
        if (sc.status != kStatusOk) break;
        if (sc.score < min_score) {
          accepted = true;
          break;
        }
        if (tid < m) sc.step[tid] *= 0.5;
        __syncthreads();
      }
      if (sc.status != kStatusOk) break;
      if (!accepted) {  // no decrease along the Gauss-Newton direction: a minimum
        converged = true;
        break;
      }
      score_red = min_score - sc.score;
      min_score = sc.score;
      if (tid < m) sc.log_sp[tid] = sc.trial[tid];
      __syncthreads();
      multi_derivatives<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
      if (tid < m) sc.gradient[tid] = sc.grad_c[tid];
      __syncthreads();
      double g2 = 0.0;  // projected gradient: a coordinate on the upper bound that V pushes outwards counts 0
      for (int r = 0; r < m; ++r)
        if (!(sc.log_sp[r] >= kGnMaxLogSp && sc.gradient[r] < 0.0)) g2 += sc.gradient[r] * sc.gradient[r];
      // a stationary point (not magic's loose stop), or V no longer moving
      // along directions that have gone flat (log lambda drifting upwards)
      if (sqrt(g2) <= kGnGradTol * (1.0 + fabs(min_score)) ||
          (score_red <= kGnFlatTol * (1.0 + min_score) && sqrt(g2) <= kGnFlatGrad * (1.0 + fabs(min_score)))) {
        converged = true;
        break;
      }
      // a decrease below kGnStallTol (1 + V): the next step is projected
      // steepest descent; a second such decrease in a row ends the search
      const bool tiny = score_red <= kGnStallTol * (1.0 + min_score);
      if (tiny && stalled) {
        converged = true;
        break;
      }
      stalled = tiny;
    }
  } else {
    for (it = 1; it <= kMaxIterations && sc.status == kStatusOk; ++it) {
      int tries = 0;
      if (it > 1) {
        if (tid < m) sc.step[tid] = steepest ? sc.steep[tid] : sc.newton[tid];
        __syncthreads();
        bool trying = true;
        while (trying) {
          ++tries;
          if (tries == 4 && !steepest) {
            steepest = true;
            if (tid < m) sc.step[tid] = sc.steep[tid];
          }
          __syncthreads();
          if (tid < m) sc.trial[tid] = sc.log_sp[tid] + sc.step[tid];
          __syncthreads();
          multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
          ++calls;
          if (sc.status != kStatusOk) break;
          const double tscore = sc.score;
          if (tscore < min_score) {
            trying = false;
            score_red = min_score - tscore;
            min_score = tscore;
            if (tid < m) sc.log_sp[tid] = sc.trial[tid];
            __syncthreads();
            multi_derivatives<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
          } else {
            if (tid < m) sc.step[tid] *= 0.5;
          }
          if (tries == max_half - 1 && trying)
            if (tid < m) sc.step[tid] = 0.0;
          if (tries == max_half) trying = false;
          __syncthreads();
        }
        if (sc.status != kStatusOk) break;
      }
      if (it > 3) {
        double g2 = 0.0;
        for (int r = 0; r < m; ++r) g2 += sc.gradient[r] * sc.gradient[r];
        converged = score_red <= kConvTol * (1.0 + min_score) &&
                    sqrt(g2) <= pow(kConvTol, 1.0 / 3.0) * (1.0 + fabs(min_score));
        if (tries == max_half) converged = true;
      }
      __syncthreads();
      if (tid == 0) {
        for (int r = 0; r < m; ++r) sc.gradient[r] = sc.grad_c[r];
        bool st = false;
        newton_from_hessian(m, &sc, &st);
        ctl[0] = st ? 1 : 0;
      }
      __syncthreads();
      steepest = ctl[0] != 0;
      if (converged) break;
    }
  }
  if (sc.status == kStatusOk && !converged) {
    __syncthreads();
    if (tid == 0) sc.status = kStatusNotConverged;
    __syncthreads();
  }
  if (sc.status == kStatusOk && selection != FKPC_SELECT_GN_NEWTON) {  // magic's boundary probes
    for (int c = 0; c < m; ++c) {
      const double direction = sc.gradient[c] < 0.0 ? 1.0 : -1.0;
      for (int probe = 0; probe < 5; ++probe) {
        if (tid < m) sc.trial[tid] = sc.log_sp[tid] + (tid == c ? direction * 2.0 : 0.0);
        __syncthreads();
        multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
        ++calls;
        if (sc.status != kStatusOk || !(sc.score < min_score)) break;
        min_score = sc.score;
        if (tid < m) sc.log_sp[tid] = sc.trial[tid];
        __syncthreads();
      }
      if (sc.status != kStatusOk) break;
    }
  }
  // terminal Newton polish from the selected point
  if (sc.status == kStatusOk) {
    __syncthreads();
    if (tid < m) sc.trial[tid] = sc.log_sp[tid];
    __syncthreads();
    multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
    for (int ps = 0; ps < kPolishSteps && sc.status == kStatusOk; ++ps) {
      multi_derivatives<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
      if (tid == 0) ctl[1] = polish_step(m, &sc);
      __syncthreads();
      const int act = ctl[1];
      if (act == 0) break;
      if (tid < m) sc.trial[tid] = sc.log_sp[tid];
      __syncthreads();
      multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
      ++calls;
      if (act == 2) break;
    }
  }
  // final fit at the selected point (the last core call may be a rejected probe)
  if (sc.status == kStatusOk) {
    __syncthreads();
    if (tid < m) sc.trial[tid] = sc.log_sp[tid];
    __syncthreads();
    multi_core<QMAX, RMAX, S, D>(des, arena, n, sm, &sc);
  }
  const double* Wg = sm + L::WG;
  double* r = residuals + static_cast<int64_t>(n) * job.out;
  const bool ok = sc.status == kStatusOk;
  for (int i = tid; i < n; i += NT) {
    double f = 0.0;
    if (ok)
      for (int c = 0; c < q; ++c) f += Q[i + static_cast<int64_t>(n) * c] * Wg[c];
    r[i] = ok ? y[i] - f : NAN;
  }
  if (tid == 0)
    store_result(results + t, sc.log_sp, m, sc.score, sc.edf, sc.rss, sc.status, it, calls,
                 sc.dropped > 0 ? kFitRankTruncated : 0);
  if (all_log_sp)
    for (int j = tid; j < kMaxPenalties; j += NT) all_log_sp[j] = j < m ? sc.log_sp[j] : NAN;
}

template <int QMAX, int RMAX>
__global__ void __launch_bounds__(kMultiThreads, 1) fit_multi_kernel(
    const DesignDev* __restrict__ designs, const double* __restrict__ arena, const double* __restrict__ data,
    int n, const FitJob* __restrict__ jobs, const int* __restrict__ job_index, int job_count,
    double* __restrict__ residuals, FitResult* __restrict__ results, int selection, double* __restrict__ workspace) {
  using L = MultiLayout<QMAX, RMAX>;
  extern __shared__ double smem_dyn[];
  // the q <= 112 class keeps its (~330 KB) working set in a global workspace per CTA
  double* sm = workspace ? workspace + static_cast<int64_t>(blockIdx.x) * L::TOTAL : smem_dyn;
  __shared__ MultiScalars sc;
  __shared__ int ctl[4];
  if (blockIdx.x >= job_count) return;
  const int t = job_index[blockIdx.x];
  const FitJob job = jobs[t];
  multi_fit_job<QMAX, RMAX, MultiScalars, DesignDev>(designs[job.design], job, t, arena, data, n, residuals, results,
                                                    selection, sm, sc, ctl, nullptr);
}

// The wide class: |S| up to 62 (q <= kWideQ, stacked roots <= kWideR rows),
// working set and scalars in a global workspace per CTA, one persistent CTA
// per SM at most walking the class's jobs.  Each design's full descriptor
// sits in the arena at its header's ``ext``; the k-th job of the class writes
// all its log(lambda) to wide_log_sp[k * kMaxPenalties ...].
constexpr int kWideThreads = 256;
using WideScalars = MultiScalarsT<kMaxPenalties, kWideThreads, kWideQ, kWideR>;
constexpr int64_t kWideScalarDoubles = static_cast<int64_t>((sizeof(WideScalars) + 15) / 16 * 2);
constexpr int64_t kWideSlotDoubles = MultiLayout<kWideQ, kWideR>::TOTAL + kWideScalarDoubles;

__global__ void __launch_bounds__(kWideThreads, 1) fit_multi_wide_kernel(
    const DesignDev* __restrict__ designs, const double* __restrict__ arena, const double* __restrict__ data,
    int n, const FitJob* __restrict__ jobs, const int* __restrict__ job_index, int job_count,
    double* __restrict__ residuals, FitResult* __restrict__ results, int selection, double* __restrict__ workspace,
    double* __restrict__ wide_log_sp) {
  using L = MultiLayout<kWideQ, kWideR>;
  __shared__ int ctl[4];
  double* sm = workspace + static_cast<int64_t>(blockIdx.x) * kWideSlotDoubles;
  WideScalars& sc = *reinterpret_cast<WideScalars*>(sm + L::TOTAL);
  for (int k = blockIdx.x; k < job_count; k += gridDim.x) {
    __syncthreads();  // the previous job's scalars are read no more
    const int t = job_index[k];
    const FitJob job = jobs[t];
    const WideDesign& des = *reinterpret_cast<const WideDesign*>(arena + designs[job.design].ext);
    multi_fit_job<kWideQ, kWideR, WideScalars, WideDesign>(des, job, t, arena, data, n, residuals, results, selection,
                                                           sm, sc, ctl, wide_log_sp + static_cast<int64_t>(k) * kMaxPenalties);
  }
}

// ------------------------------------------------------ multi, warp per fit
//
// fit_multi_warp_kernel: one warp per target for the additive designs of the
// warp class (q <= kWarpQ, rsum <= kWarpR, m <= kWarpM: |S| = 3 and 4 with
// k = 10 margins).  The evaluation and the Newton loop are those of
// fit_multi_kernel, laid out so that no step waits on a block barrier, many
// fits share an SM, and the code the warps run stays small enough for the
// instruction cache (every phase is a short loop, nothing is unrolled over
// the coefficient index):
//  - fold: lane j keeps column j of the stacked roots in registers (columns
//    32..39 in a second register slot of lanes 0..7 until the first q - 32
//    pivots are done, then moved into the first slot); the pivot lane
//    publishes its column and reflector through shared memory and every lane
//    updates its own column, rows < nzrow(k) only;
//  - W = R Ra^-1 (lane = row of W) and T = Ra^-T root (lane = column of T)
//    are right-looking forward substitutions in shared memory, the rows of
//    Ra read as broadcasts;
//  - C = T'T and D = (WT)'(WT): lane a accumulates row a of both over the
//    coefficient index, reading rows of T and WT as broadcasts, then forms
//    the four block sums the Hessian needs per pair of penalty blocks; a
//    final pass sums them over the lanes of each block.
namespace {

constexpr int kWarpPart = 19;  // per-lane partial sums (odd stride)
constexpr int kWarpSums = 4 * kWarpM * kWarpM + 2 * kWarpM;

struct WarpLayout {
  static constexpr int X = 0;                    // Ra (packed rows) | WT (row-major) | per-lane partials
  static constexpr int XSZ = kWarpQ * kWarpR;
  static constexpr int Y = X + XSZ;              // W (packed rows)
  static constexpr int Z = Y + kWarpTri;         // T (row-major) | block sums, Newton scratch
  static constexpr int Y0 = Z + XSZ;
  static constexpr int G = Y0 + kWarpQ;
  static constexpr int WG = G + kWarpQ;
  static constexpr int E1 = WG + kWarpQ;
  static constexpr int IDG = E1 + kWarpQ;
  static constexpr int AV = IDG + kWarpQ;
  static constexpr int BV = AV + kWarpR;
  static constexpr int PV = BV + kWarpR;         // pivot column of the fold
  static constexpr int TOTAL = PV + kWarpR;
};
static_assert(WarpLayout::XSZ >= kWarpTri && WarpLayout::XSZ >= 32 * kWarpPart, "warp layout");
static_assert(WarpLayout::XSZ >= kWarpSums + 2 * kWarpM * kWarpM, "warp layout");
static_assert(kWarpR == 32 && kWarpQ > 32 && kWarpQ <= 64 && kWarpQ % 4 == 0, "warp class shape");
static_assert(kWarpTri % 2 == 0 && WarpLayout::Y % 2 == 0, "16-byte copies of the packed triangle");

struct WarpScalars {
  static constexpr int kLd = kWarpM;  // leading dimension of the m x m matrices
  double beta, v0, score, rss, edf, rss0;  // rss0 = |y - Q Q'y|^2
  double dmax;                              // largest pivot of the current fold
  int dropped;                              // coefficients the rank rule dropped at the last evaluation
  double lam[kWarpM];
  double log_sp[kWarpM];
  double trial[kWarpM];
  double step[kWarpM];
  double grad_c[kWarpM];
  double gradient[kWarpM];
  double newton[kWarpM];
  double steep[kWarpM];
  double ddelta[kWarpM];
  double drss[kWarpM];
  double hess_c[kWarpM * kWarpM];
  double gn_c[kWarpM * kWarpM];  // Gauss-Newton Hessian (adjoint entry point)
  double* ja;  // Newton scratch (Cholesky factor / Jacobi matrix), in the Z region
  double* jv;  // Jacobi rotations, in the Z region
  int status;
  int ctl;
  int nzrow[kWarpQ];
  int rowblk[kWarpR];  // penalty block of each stacked root row (-1 beyond rsum)
};

// Per-warp state of the warp kernels: one slot of dynamic shared memory per
// warp (work arrays, scalars, design descriptor), addressed from the file-scope
// array so that the out-of-line evaluation and derivative routines keep
// shared-memory addressing.
extern __shared__ __align__(16) double s_warp_dyn[];
constexpr int kWarpScalarDoubles = static_cast<int>((sizeof(WarpScalars) + 7) / 8);
constexpr int kWarpDesignDoubles = static_cast<int>((sizeof(WarpDesign) + 7) / 8);
constexpr int kWarpSlotDoubles = (WarpLayout::TOTAL + kWarpScalarDoubles + kWarpDesignDoubles + 1) & ~1;
constexpr size_t kWarpSlotBytes = sizeof(double) * kWarpSlotDoubles;

__device__ __forceinline__ double* warp_slot() { return s_warp_dyn + (threadIdx.x >> 5) * kWarpSlotDoubles; }
__device__ __forceinline__ WarpScalars& warp_scalars() {
  return *reinterpret_cast<WarpScalars*>(warp_slot() + WarpLayout::TOTAL);
}
__device__ __forceinline__ WarpDesign& warp_design() {
  return *reinterpret_cast<WarpDesign*>(warp_slot() + WarpLayout::TOTAL + kWarpScalarDoubles);
}

// The warp-class descriptor (m <= kWarpM) from the full one, lanes in parallel.
__device__ __forceinline__ void copy_warp_design(const DesignDev* __restrict__ d, int lane) {
  WarpDesign& w = warp_design();
  if (lane == 0) {
    w.kind = d->kind;
    w.q = d->q;
    w.m = d->m;
    w.rsum = d->rsum;
    w.basis = d->basis;
    w.rmat = d->rmat;
    w.spec = d->spec;
    w.roots = d->roots;
    w.rpack = d->rpack;
  }
  if (lane < kWarpM) {
    w.off[lane] = d->off[lane];
    w.dim[lane] = d->dim[lane];
    w.rank[lane] = d->rank[lane];
    w.rowoff[lane] = d->rowoff[lane];
    w.rootoff[lane] = d->rootoff[lane];
    w.log_sp0[lane] = d->log_sp0[lane];
  }
}

// Asynchronous 16-byte global -> shared copies (cp.async, L1-allocating).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Column ``col`` of the stacked roots scaled by sqrt(lambda) (rows 0..kWarpR-1).
__device__ __forceinline__ void warp_root_column(const WarpDesign& des, const double* __restrict__ arena,
                                                 const WarpScalars& sc, int col, int jb, double (&b)[kWarpR]) {
  int ro = 0, rk = 0, dim = 1, a = 0;
  double s = 0.0;
  const double* root = arena + des.roots;
  if (jb >= 0) {
    ro = des.rowoff[jb];
    rk = des.rank[jb];
    dim = des.dim[jb];
    a = col - des.off[jb];
    s = sqrt(sc.lam[jb]);
    root += des.rootoff[jb];
  }
#pragma unroll
  for (int r = 0; r < kWarpR; ++r) b[r] = (r >= ro && r < ro + rk) ? s * root[a + dim * (r - ro)] : 0.0;
}

// Apply the step-k reflector (pv, v0, beta) to this lane's column ``col``.
__device__ __forceinline__ void warp_fold_update(int k, int q, int nz, double beta, double v0, double* X,
                                                 const double* pv, double (&b)[kWarpR], int col) {
  if (col > k && col < q) {
    const double2* p2 = reinterpret_cast<const double2*>(pv);
    const int at = packed_row(k, col);
    double w0 = v0 * X[at], w1 = 0.0, w2 = 0.0, w3 = 0.0;
#pragma unroll
    for (int h = 0; h < kWarpR / 8; ++h) {
      if (8 * h < nz) {
#pragma unroll
        for (int u = 0; u < 8; u += 4) {
          const int r = 8 * h + u;
          const double2 pa = p2[r / 2], pb = p2[r / 2 + 1];
          w0 += pa.x * b[r];
          w1 += pa.y * b[r + 1];
          w2 += pb.x * b[r + 2];
          w3 += pb.y * b[r + 3];
        }
      }
    }
    const double w = beta * ((w0 + w1) + (w2 + w3));
    X[at] -= w * v0;
#pragma unroll
    for (int h = 0; h < kWarpR / 8; ++h) {
      if (8 * h < nz) {
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
          const int r = 8 * h + u;
          const double2 pa = p2[r / 2];
          b[r] -= w * pa.x;
          b[r + 1] -= w * pa.y;
        }
      }
    }
  }
}

// Step k of the fold.  The pivot column k sits in slot 0 of lane k & 31; its
// rows >= nzrow(k) are exactly zero, so only the 8-row chunks below nz count.
template <bool TWO>
__device__ __forceinline__ void warp_fold_step(int k, int q, WarpScalars& sc, double* X, double* pv,
                                               double (&b0)[kWarpR], double (&b1)[kWarpR], int col0, int col1) {
  const int lane = threadIdx.x & 31;
  const int nz = sc.nzrow[k];
  if (lane == (k & 31)) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    double2* p2 = reinterpret_cast<double2*>(pv);
#pragma unroll
    for (int h = 0; h < kWarpR / 8; ++h) {
      if (8 * h < nz) {
#pragma unroll
        for (int u = 0; u < 8; u += 4) {
          const int r = 8 * h + u;
          s0 += b0[r] * b0[r];
          s1 += b0[r + 1] * b0[r + 1];
          s2 += b0[r + 2] * b0[r + 2];
          s3 += b0[r + 3] * b0[r + 3];
          p2[r / 2] = make_double2(b0[r], b0[r + 1]);
          p2[r / 2 + 1] = make_double2(b0[r + 2], b0[r + 3]);
        }
      }
    }
    const double sg = (s0 + s1) + (s2 + s3);
    const int kk = packed_row(k, k);
    const double akk = X[kk];
    double beta = 0.0, v0 = 0.0, piv = fabs(akk);
    if (sg != 0.0) {
      const double nrm = sqrt(akk * akk + sg);
      const double alpha = akk >= 0.0 ? -nrm : nrm;
      v0 = akk - alpha;
      beta = 2.0 / (v0 * v0 + sg);
      X[kk] = alpha;
      piv = nrm;
    }
    sc.dmax = fmax(sc.dmax, piv);  // the largest pivot so far, for the rank rule
    sc.beta = beta;
    sc.v0 = v0;
  }
  __syncwarp();
  const double beta = sc.beta;
  const double v0 = sc.v0;
  if (beta != 0.0) {
    warp_fold_update(k, q, nz, beta, v0, X, pv, b0, col0);
    if (TWO) warp_fold_update(k, q, nz, beta, v0, X, pv, b1, col1);
  }
  __syncwarp();
}

// Left-looking forward substitution through Ra' on one shared-memory vector
// ``v`` of stride ``ld`` (v[ld * c] is entry c, holding the right-hand side):
// for c = start..q-1, v[c] = (v[c] - sum_{s in [start, c)} v[s] Ra(s, c)) / Ra(c, c).
// Each entry is one dot product with four chains, so its loads overlap.
// Returns the sum of squares of the solved entries.
__device__ __forceinline__ double warp_left_subst(double* __restrict__ v, int ld, int start, int q,
                                                  const double* __restrict__ Ra, const double* __restrict__ idg) {
  double ss = 0.0;
  for (int c = start; c < q; ++c) {
    double s0 = v[ld * c], s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int t = start;
    for (; t + 3 < c; t += 4) {
      s0 -= v[ld * t] * Ra[packed_row(t, c)];
      s1 -= v[ld * (t + 1)] * Ra[packed_row(t + 1, c)];
      s2 -= v[ld * (t + 2)] * Ra[packed_row(t + 2, c)];
      s3 -= v[ld * (t + 3)] * Ra[packed_row(t + 3, c)];
    }
    for (; t < c; ++t) s0 -= v[ld * t] * Ra[packed_row(t, c)];
    const double w = ((s0 + s1) + (s2 + s3)) * idg[c];
    v[ld * c] = w;
    ss += w * w;
  }
  return ss;
}

// Dot product of a[0..len) (stride 1) with b[0..len) (stride ldb), four chains.
__device__ __forceinline__ double warp_dot(const double* __restrict__ a, const double* __restrict__ b, int ldb,
                                           int len) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int i = 0;
  for (; i + 3 < len; i += 4) {
    s0 = fma(a[i], b[ldb * i], s0);
    s1 = fma(a[i + 1], b[ldb * (i + 1)], s1);
    s2 = fma(a[i + 2], b[ldb * (i + 2)], s2);
    s3 = fma(a[i + 3], b[ldb * (i + 3)], s3);
  }
  for (; i < len; ++i) s0 = fma(a[i], b[ldb * i], s0);
  return (s0 + s1) + (s2 + s3);
}

// sum_{i <= c} W(i, c) v[i] for the row-packed W, four chains.
__device__ __forceinline__ double warp_column_dot(const double* __restrict__ W, int c, const double* __restrict__ v) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int i = 0;
  for (; i + 3 <= c; i += 4) {
    s0 += W[packed_row(i, c)] * v[i];
    s1 += W[packed_row(i + 1, c)] * v[i + 1];
    s2 += W[packed_row(i + 2, c)] * v[i + 2];
    s3 += W[packed_row(i + 3, c)] * v[i + 3];
  }
  for (; i <= c; ++i) s0 += W[packed_row(i, c)] * v[i];
  return (s0 + s1) + (s2 + s3);
}

// Objective at sc.trial.  Leaves Ra in X and W in Y (row-packed, valid for
// columns < q), idg, g, Wg and score / rss / edf in sc.
__device__ __noinline__ void warp_core(const double* __restrict__ arena, int n, int jb0, int jb1) {
  using L = WarpLayout;
  const WarpDesign& des = warp_design();
  WarpScalars& sc = warp_scalars();
  double* sm = warp_slot();
  const int lane = threadIdx.x & 31;
  const int q = des.q;
  double* X = sm + L::X;
  double* Y = sm + L::Y;
  double* pv = sm + L::PV;
  double* idg = sm + L::IDG;
  if (lane < des.m) sc.lam[lane] = exp(sc.trial[lane]);
  {
    // R (row-packed) into X, where the fold turns it into Ra, and into Y,
    // where the W solve starts from it; only the first copy is waited for
    // before the fold.
    const double* rpack = arena + des.rpack;
    for (int idx = 2 * lane; idx < kWarpTri; idx += 64) cp_async16(X + idx, rpack + idx);
    cp_async_commit();
    for (int idx = 2 * lane; idx < kWarpTri; idx += 64) cp_async16(Y + idx, rpack + idx);
    cp_async_commit();
    cp_async_wait<1>();
  }
  if (lane == 0) sc.dmax = 0.0;
  __syncwarp();
  {
    double b0[kWarpR], b1[kWarpR];
    warp_root_column(des, arena, sc, lane, jb0, b0);
    if (q > 32) warp_root_column(des, arena, sc, lane + 32, jb1, b1);
    int col0 = lane;
    const int qa = q - 32;
    for (int k = 0; k < qa; ++k) warp_fold_step<true>(k, q, sc, X, pv, b0, b1, col0, lane + 32);
    if (lane < qa) {
#pragma unroll
      for (int r = 0; r < kWarpR; ++r) b0[r] = b1[r];
      col0 = lane + 32;
    }
    for (int k = qa > 0 ? qa : 0; k < q; ++k) warp_fold_step<false>(k, q, sc, X, pv, b0, b1, col0, 0);
  }
  {
    // the rank rule drops the coefficients of negligible pivots (the fold
    // kept the largest pivot in sc.dmax)
    const double tol = kRankTol * sc.dmax;
    int dropped = 0;
    for (int c0 = 0; c0 < q; c0 += 32) {
      const int c = c0 + lane;
      bool drop = false;
      if (c < q) {
        const double d = X[packed_row(c, c)];
        drop = !(fabs(d) > tol);
        idg[c] = drop ? 0.0 : 1.0 / d;
      }
      dropped += __popc(__ballot_sync(0xffffffffu, drop));
    }
    if (lane == 0) {
      sc.dropped = dropped;
      if (!(sc.dmax > 0.0)) sc.status = kStatusRank;
    }
  }
  // W = R Ra^-1: row i (lane i; rows 32.. on lanes 0..) solves w Ra = R(i, :).
  // Packed row i starts at Y + packed_row(i, 0), entry c >= i at offset c.
  cp_async_wait<0>();
  __syncwarp();
  double e = 0.0;
  for (int i = lane; i < q; i += 32) e += warp_left_subst(Y + packed_row(i, 0), 1, i, q, X, idg);
  const double edf = warp_sum(e);
  __syncwarp();
  const double* y0 = sm + L::Y0;
  double* g = sm + L::G;
  double* wg = sm + L::WG;
  for (int c = lane; c < q; c += 32) g[c] = warp_column_dot(Y, c, y0);
  __syncwarp();
  // RSS = |y - Q y0|^2 + |y0 - W g|^2: sums of squares, no cancellation
  double gg = 0.0;
  for (int i = lane; i < q; i += 32) {
    const double s = warp_dot(Y + packed_row(i, 0) + i, g + i, 1, q - i);
    wg[i] = s;
    const double d = y0[i] - s;
    gg += d * d;
  }
  const double part = warp_sum(gg);
  if (lane == 0) {
    const double rss = sc.rss0 + part;
    const double delta = static_cast<double>(n) - edf;
    sc.rss = rss;
    sc.edf = edf;
    if (!(isfinite(rss) && isfinite(edf)) || delta <= 1e-8) {
      sc.score = INFINITY;
      if (sc.status == kStatusOk) sc.status = kStatusNumeric;
    } else {
      sc.score = static_cast<double>(n) * rss / (delta * delta);
    }
  }
  __syncwarp();
}

// C = T'T and D = (WT)'(WT) for the 16 columns b = B0..B0+15: row a (this
// lane) accumulated over the coefficient index, then folded into the block
// sums p[bj] = {sum C.D, sum D a_b, sum C a_b, sum C b_b} over b in block bj.
// Column b's terms of the block sums, from C(a, b) and D(a, b) of this lane's
// row a; explicit roundings, so that every path that forms the block sums in
// the same order of b gets the same bits.
__device__ __forceinline__ void block_term(int b, double c, double d, const double* av, const double* bv,
                                           const WarpScalars& sc, double (&p)[kWarpM][4]) {
  const int jb = sc.rowblk[b];
  const double avb = av[b], bvb = bv[b];
  const double cd = __dmul_rn(c, d), da = __dmul_rn(d, avb), ca = __dmul_rn(c, avb), cb = __dmul_rn(c, bvb);
#pragma unroll
  for (int bj = 0; bj < kWarpM; ++bj)
    if (jb == bj) {
      p[bj][0] = __dadd_rn(p[bj][0], cd);
      p[bj][1] = __dadd_rn(p[bj][1], da);
      p[bj][2] = __dadd_rn(p[bj][2], ca);
      p[bj][3] = __dadd_rn(p[bj][3], cb);
    }
}

template <int B0>
__device__ __forceinline__ void warp_block_sums(int q, const double* WT, const double* T, const double* av,
                                                const double* bv, const WarpScalars& sc, double (&p)[kWarpM][4]) {
  const int lane = threadIdx.x & 31;
  double c[16], d[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) c[u] = d[u] = 0.0;
  for (int i = 0; i < q; ++i) {
    const double ta = T[kWarpR * i + lane];
    const double wa = WT[kWarpR * i + lane];
    const double2* trow = reinterpret_cast<const double2*>(T + kWarpR * i + B0);
    const double2* wrow = reinterpret_cast<const double2*>(WT + kWarpR * i + B0);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double2 x = trow[u], y = wrow[u];
      c[2 * u] = fma(ta, x.x, c[2 * u]);
      c[2 * u + 1] = fma(ta, x.y, c[2 * u + 1]);
      d[2 * u] = fma(wa, y.x, d[2 * u]);
      d[2 * u + 1] = fma(wa, y.y, d[2 * u + 1]);
    }
  }
#pragma unroll
  for (int u = 0; u < 16; ++u) block_term(B0 + u, c[u], d[u], av, bv, sc, p);
}

// Gradient and Hessian of V at the point of the last warp_core call (the
// quantities of multi_derivatives), in three pieces on a warp slot ``sm``:
// deriv_setup (one warp): e1 = g - W'(W g), T = Ra^-T root (lane a: column a,
// row-major in Z), a = T'g and b = T'e1 into AV / BV; then WT = W T into X,
// the per-lane sum of squares of WT and the block sums of C = T'T and
// D = (WT)'(WT) (warp_derivatives on one warp, spec_derivatives on the
// continuation's warps); deriv_finish (one warp): the partial sums, the
// gradient and both Hessians.  jrow: penalty block of stacked row ``lane``.
__device__ __forceinline__ void deriv_setup(double* sm, const double* __restrict__ arena, int jrow) {
  using L = WarpLayout;
  const WarpDesign& des = *reinterpret_cast<const WarpDesign*>(sm + L::TOTAL + kWarpScalarDoubles);
  const int lane = threadIdx.x & 31;
  const int q = des.q;
  double* X = sm + L::X;
  const double* Y = sm + L::Y;
  double* Z = sm + L::Z;
  const double* g = sm + L::G;
  const double* wg = sm + L::WG;
  double* e1 = sm + L::E1;
  const double* idg = sm + L::IDG;
  double* av = sm + L::AV;
  double* bv = sm + L::BV;
  // e1 = g - W'(W g)
  for (int c = lane; c < q; c += 32) e1[c] = g[c] - warp_column_dot(Y, c, wg);
  // T(:, a) = Ra^-T root(:, a): lane a, column a of Z (row-major, stride kWarpR)
  double* ta = Z + lane;
  {
    int off = 0, dim = 0, cc = 0;
    const double* root = arena + des.roots;
    if (jrow >= 0) {
      off = des.off[jrow];
      dim = des.dim[jrow];
      cc = lane - des.rowoff[jrow];
      root += des.rootoff[jrow];
    }
    for (int i = 0; i < q; ++i) ta[kWarpR * i] = 0.0;
    for (int i0 = 0; i0 < dim; i0 += 16) {
      double r[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) r[u] = i0 + u < dim ? root[i0 + u + dim * cc] : 0.0;
#pragma unroll
      for (int u = 0; u < 16; ++u)
        if (i0 + u < dim) ta[kWarpR * (off + i0 + u)] = r[u];
    }
  }
  if (jrow >= 0) warp_left_subst(ta, kWarpR, des.off[jrow], q, X, idg);
  __syncwarp();  // e1 written; every read of Ra done: X may take WT
  av[lane] = warp_dot(g, ta, kWarpR, q);
  bv[lane] = warp_dot(e1, ta, kWarpR, q);
  __syncwarp();
}

__device__ __forceinline__ void deriv_finish(double* sm, int n, double (&p)[kWarpM][4], double dd) {
  using L = WarpLayout;
  const WarpDesign& des = *reinterpret_cast<const WarpDesign*>(sm + L::TOTAL + kWarpScalarDoubles);
  WarpScalars& sc = *reinterpret_cast<WarpScalars*>(sm + L::TOTAL);
  const int lane = threadIdx.x & 31;
  const int m = des.m;
  double* X = sm + L::X;
  double* Z = sm + L::Z;
  const double sa = sm[L::AV + lane], sb = sm[L::BV + lane];
  __syncwarp();  // T / WT reads done: X takes the per-lane partial sums
  {
    double* part = X + kWarpPart * lane;
#pragma unroll
    for (int bj = 0; bj < kWarpM; ++bj) {
      part[4 * bj + 0] = p[bj][0];
      part[4 * bj + 1] = p[bj][1] * sa;  // a_j' D_ji a_i
      part[4 * bj + 2] = p[bj][2] * sb;  // b_i' C_ij a_j
      part[4 * bj + 3] = p[bj][3] * sa;  // b_j' C_ji a_i
    }
    part[4 * kWarpM] = dd;
    part[4 * kWarpM + 1] = sb * sa;
  }
  __syncwarp();
  double* hsum = Z;  // T is no longer needed
  for (int o = lane; o < kWarpSums; o += 32) {
    int bi, slot;
    if (o < 4 * kWarpM * kWarpM) {
      bi = o / (4 * kWarpM);
      slot = o % (4 * kWarpM);
      if (slot / 4 >= m) bi = kWarpM;
    } else {
      bi = (o - 4 * kWarpM * kWarpM) / 2;
      slot = 4 * kWarpM + (o - 4 * kWarpM * kWarpM) % 2;
    }
    double s = 0.0;
    if (bi < m)
      for (int a = des.rowoff[bi]; a < des.rowoff[bi] + des.rank[bi]; ++a) s += X[kWarpPart * a + slot];
    hsum[o] = s;
  }
  __syncwarp();
  if (lane == 0) {
    const double nd = static_cast<double>(n);
    const double delta = nd - sc.edf;
    const double s1 = nd / (delta * delta);
    const double s2 = 2.0 * s1 * sc.rss / delta;
    for (int j = 0; j < m; ++j) {
      sc.ddelta[j] = sc.lam[j] * hsum[4 * kWarpM * kWarpM + 2 * j];
      sc.drss[j] = 2.0 * sc.lam[j] * hsum[4 * kWarpM * kWarpM + 2 * j + 1];
    }
    for (int bi = 0; bi < m; ++bi)
      for (int bj = 0; bj <= bi; ++bj) {
        const double* hs = hsum + 4 * kWarpM * bi + 4 * bj;
        const double ll = sc.lam[bi] * sc.lam[bj];
        double d2delta = -2.0 * ll * hs[0];
        double d2rss = 2.0 * ll * (hs[1] - hs[2] - hs[3]);
        if (bi == bj) {
          d2delta += sc.ddelta[bi];
          d2rss += sc.drss[bi];
        }
        const double h = -2.0 * s1 / delta * (sc.ddelta[bj] * sc.drss[bi] + sc.ddelta[bi] * sc.drss[bj]) +
                         s1 * d2rss + 3.0 * s2 / delta * sc.ddelta[bi] * sc.ddelta[bj] - s2 * d2delta;
        sc.hess_c[bi + WarpScalars::kLd * bj] = h;
        sc.hess_c[bj + WarpScalars::kLd * bi] = h;
        // Gauss-Newton: V = |f|^2, f = sqrt(n) r / delta, dr_i . dr_j = ll a_i' D_ij a_j
        const double gn = 2.0 * s1 * ll * hs[1] -
                          s1 / delta * (sc.ddelta[bj] * sc.drss[bi] + sc.ddelta[bi] * sc.drss[bj]) +
                          s2 / delta * sc.ddelta[bi] * sc.ddelta[bj];
        sc.gn_c[bi + WarpScalars::kLd * bj] = gn;
        sc.gn_c[bj + WarpScalars::kLd * bi] = gn;
      }
    for (int j = 0; j < m; ++j) sc.grad_c[j] = s1 * sc.drss[j] - s2 * sc.ddelta[j];
  }
  __syncwarp();
}

__device__ __noinline__ void warp_derivatives(const double* __restrict__ arena, int n, int jrow) {
  using L = WarpLayout;
  double* sm = warp_slot();
  const WarpDesign& des = warp_design();
  const WarpScalars& sc = warp_scalars();
  const int lane = threadIdx.x & 31;
  const int q = des.q;
  double* X = sm + L::X;
  const double* Y = sm + L::Y;
  const double* Z = sm + L::Z;
  deriv_setup(sm, arena, jrow);
  // WT(:, a) = W T(:, a), row-major in X
  const double* ta = Z + lane;
  double dd = 0.0;
  for (int i = 0; i < q; ++i) {
    const double s = warp_dot(Y + packed_row(i, 0) + i, ta + kWarpR * i, kWarpR, q - i);
    X[kWarpR * i + lane] = s;
    dd = fma(s, s, dd);
  }
  __syncwarp();
  double p[kWarpM][4];
#pragma unroll
  for (int bj = 0; bj < kWarpM; ++bj) p[bj][0] = p[bj][1] = p[bj][2] = p[bj][3] = 0.0;
  warp_block_sums<0>(q, X, Z, sm + L::AV, sm + L::BV, sc, p);
  warp_block_sums<16>(q, X, Z, sm + L::AV, sm + L::BV, sc, p);
  deriv_finish(sm, n, p, dd);
}

}  // namespace

// Per-fit set-up shared by the fit and adjoint kernels: the design
// descriptor into shared memory, fill-in bounds and block maps, y0 = Q'y and
// |y|^2.  Returns the penalty blocks of this lane's columns and stacked row.
__device__ __noinline__ void warp_fit_setup(const DesignDev* __restrict__ design, const double* __restrict__ arena,
                                            const double* __restrict__ y, int n, int* jb0_out, int* jb1_out,
                                            int* jrow_out) {
  using L = WarpLayout;
  double* sm = warp_slot();
  WarpScalars& sc = warp_scalars();
  const WarpDesign& des = warp_design();
  const int lane = threadIdx.x & 31;
  copy_warp_design(design, lane);
  if (lane == 0) {
    sc.status = kStatusOk;
    sc.ja = sm + L::Z + kWarpSums;
    sc.jv = sc.ja + WarpScalars::kLd * WarpScalars::kLd;
  }
  __syncwarp();
  const int q = des.q, m = des.m;
  int jb0 = -1, jb1 = -1, jrow = -1;
  for (int j = 0; j < m; ++j) {
    if (lane < q && lane >= des.off[j] && lane < des.off[j] + des.dim[j]) jb0 = j;
    if (lane + 32 < q && lane + 32 >= des.off[j] && lane + 32 < des.off[j] + des.dim[j]) jb1 = j;
    if (lane >= des.rowoff[j] && lane < des.rowoff[j] + des.rank[j]) jrow = j;
  }
  sc.rowblk[lane] = jrow;
  for (int c = lane; c < kWarpQ; c += 32) {
    int nz = 0;
    for (int j = 0; j < m; ++j)
      if (des.off[j] <= c) nz = des.rowoff[j] + des.rank[j];
    sc.nzrow[c] = nz;
  }
  const double* Q = arena + des.basis;
  double* y0 = sm + L::Y0;
  for (int c0 = 0; c0 < q; c0 += 4) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = lane; i < n; i += 32) {
      const double yi = y[i];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c0 + u < q) s[u] += Q[i + static_cast<int64_t>(n) * (c0 + u)] * yi;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double v = warp_sum(s[u]);
      if (lane == 0 && c0 + u < q) y0[c0 + u] = v;
    }
  }
  __syncwarp();
  {
    double ee = 0.0;  // rss0 = |y - Q y0|^2
    for (int i = lane; i < n; i += 32) {
      double f = 0.0;
      for (int c = 0; c < q; ++c) f += Q[i + static_cast<int64_t>(n) * c] * y0[c];
      const double e = y[i] - f;
      ee += e * e;
    }
    ee = warp_sum(ee);
    if (lane == 0) sc.rss0 = ee;
  }
  *jb0_out = jb0;
  *jb1_out = jb1;
  *jrow_out = jrow;
}

__global__ void __launch_bounds__(32) fit_multi_warp_kernel(const DesignDev* __restrict__ designs,
                                                            const double* __restrict__ arena,
                                                            const double* __restrict__ data, int n,
                                                            const FitJob* __restrict__ jobs,
                                                            const int* __restrict__ job_index, int job_count,
                                                            double* __restrict__ residuals,
                                                            FitResult* __restrict__ results, int selection,
                                                            int defer_calls, FitState* __restrict__ states,
                                                            int* __restrict__ defer_list,
                                                            int* __restrict__ defer_count) {
  using L = WarpLayout;
  double* sm = warp_slot();
  WarpScalars& sc = warp_scalars();
  const WarpDesign& des = warp_design();
  if (blockIdx.x >= job_count) return;
  const int lane = threadIdx.x & 31;
  const int t = job_index[blockIdx.x];
  const FitJob job = jobs[t];
  int jb0 = -1, jb1 = -1, jrow = -1;
  warp_fit_setup(designs + job.design, arena, data + static_cast<int64_t>(n) * job.column, n, &jb0, &jb1, &jrow);
  const int q = des.q, m = des.m;
  const double* y = data + static_cast<int64_t>(n) * job.column;
  const double* Q = arena + des.basis;
  if (lane < m) {
    sc.log_sp[lane] = des.log_sp0[lane];
    sc.trial[lane] = des.log_sp0[lane];
  }
  __syncwarp();
  warp_core(arena, n, jb0, jb1);
  warp_derivatives(arena, n, jrow);
  double min_score = sc.score;
  double score_red = 1e10;
  bool steepest = false;
  bool converged = false;
  int calls = 1;
  int it = 0;
  const int max_half = 25;
  if (lane < m) {
    sc.gradient[lane] = 0.0;
    sc.newton[lane] = 0.0;
    sc.steep[lane] = 0.0;
  }
  __syncwarp();
  if (selection == FKPC_SELECT_GN_NEWTON) {
    // Newton on the Gauss-Newton Hessian, halving until V decreases
    if (lane < m) sc.gradient[lane] = sc.grad_c[lane];
    __syncwarp();
    bool stalled = false;
    for (it = 1; it <= kMaxIterations && sc.status == kStatusOk; ++it) {
      if (lane == 0) {
        if (stalled) gn_steepest(m, &sc);
        else gn_step(m, &sc);
      }
      __syncwarp();
      bool accepted = false;
      for (int tries = 1; tries <= max_half; ++tries) {
        if (lane < m) sc.trial[lane] = sc.log_sp[lane] + sc.step[lane];
        __syncwarp();
        warp_core(arena, n, jb0, jb1);
        ++calls;
        if (sc.status != kStatusOk) break;
        if (sc.score < min_score) {
          accepted = true;
          break;
        }
        if (lane < m) sc.step[lane] *= 0.5;
        __syncwarp();
      }
      if (sc.status != kStatusOk) break;
      if (!accepted) {  // no decrease along the Gauss-Newton direction: a minimum
        converged = true;
        break;
      }
      score_red = min_score - sc.score;
      min_score = sc.score;
      if (lane < m) sc.log_sp[lane] = sc.trial[lane];
      __syncwarp();
      warp_derivatives(arena, n, jrow);
      if (lane < m) sc.gradient[lane] = sc.grad_c[lane];
      __syncwarp();
      double g2 = 0.0;  // projected gradient: a coordinate on the upper bound that V pushes outwards counts 0
      for (int r = 0; r < m; ++r)
        if (!(sc.log_sp[r] >= kGnMaxLogSp && sc.gradient[r] < 0.0)) g2 += sc.gradient[r] * sc.gradient[r];
      // a stationary point (not magic's loose stop), or V no longer moving
      // along directions that have gone flat (log lambda drifting upwards)
      if (sqrt(g2) <= kGnGradTol * (1.0 + fabs(min_score)) ||
          (score_red <= kGnFlatTol * (1.0 + min_score) && sqrt(g2) <= kGnFlatGrad * (1.0 + fabs(min_score)))) {
        converged = true;
        break;
      }
      // a decrease below kGnStallTol (1 + V): the next step is projected
      // steepest descent; a second such decrease in a row ends the search
      const bool tiny = score_red <= kGnStallTol * (1.0 + min_score);
      if (tiny && stalled) {
        converged = true;
        break;
      }
      stalled = tiny;
    }
  } else {
    for (it = 1; it <= kMaxIterations && sc.status == kStatusOk; ++it) {
      int tries = 0;
      if (it > 1 && defer_calls > 0 && calls >= defer_calls) {
        // a long search: hand it, at this iteration boundary, to the
        // speculative continuation kernel (several trials at once)
        FitState& st = states[t];
        if (lane < m) {
          st.log_sp[lane] = sc.log_sp[lane];
          st.newton[lane] = sc.newton[lane];
          st.steep[lane] = sc.steep[lane];
          st.gradient[lane] = sc.gradient[lane];
          for (int j = 0; j < m; ++j) st.hess[lane + kWarpM * j] = sc.hess_c[lane + WarpScalars::kLd * j];
        }
        if (lane == 0) {
          st.min_score = min_score;
          st.score_red = score_red;
          st.it = it;
          st.calls = calls;
          st.steepest = steepest ? 1 : 0;
          defer_list[atomicAdd(defer_count, 1)] = t;
        }
        return;
      }
      if (it > 1) {
        if (lane < m) sc.step[lane] = steepest ? sc.steep[lane] : sc.newton[lane];
        __syncwarp();
        bool trying = true;
        while (trying) {
          ++tries;
          if (tries == 4 && !steepest) {
            steepest = true;
            if (lane < m) sc.step[lane] = sc.steep[lane];
          }
          __syncwarp();
          if (lane < m) sc.trial[lane] = sc.log_sp[lane] + sc.step[lane];
          __syncwarp();
          warp_core(arena, n, jb0, jb1);
          ++calls;
          if (sc.status != kStatusOk) break;
          const double tscore = sc.score;
          if (tscore < min_score) {
            trying = false;
            score_red = min_score - tscore;
            min_score = tscore;
            if (lane < m) sc.log_sp[lane] = sc.trial[lane];
            __syncwarp();
            warp_derivatives(arena, n, jrow);
          } else {
            if (lane < m) sc.step[lane] *= 0.5;
          }
          if (tries == max_half - 1 && trying)
            if (lane < m) sc.step[lane] = 0.0;
          if (tries == max_half) trying = false;
          __syncwarp();
        }
        if (sc.status != kStatusOk) break;
      }
      if (it > 3) {
        double g2 = 0.0;
        for (int r = 0; r < m; ++r) g2 += sc.gradient[r] * sc.gradient[r];
        converged = score_red <= kConvTol * (1.0 + min_score) &&
                    sqrt(g2) <= pow(kConvTol, 1.0 / 3.0) * (1.0 + fabs(min_score));
        if (tries == max_half) converged = true;
      }
      __syncwarp();
      if (lane == 0) {
        for (int r = 0; r < m; ++r) sc.gradient[r] = sc.grad_c[r];
        bool st = false;
        newton_from_hessian(m, &sc, &st);
        sc.ctl = st ? 1 : 0;
      }
      __syncwarp();
      steepest = sc.ctl != 0;
      if (converged) break;
    }
  }
  if (sc.status == kStatusOk && !converged) {
    __syncwarp();
    if (lane == 0) sc.status = kStatusNotConverged;
    __syncwarp();
  }
  if (sc.status == kStatusOk && selection != FKPC_SELECT_GN_NEWTON) {  // magic's boundary probes
    for (int c = 0; c < m; ++c) {
      const double direction = sc.gradient[c] < 0.0 ? 1.0 : -1.0;
      for (int probe = 0; probe < 5; ++probe) {
        if (lane < m) sc.trial[lane] = sc.log_sp[lane] + (lane == c ? direction * 2.0 : 0.0);
        __syncwarp();
        warp_core(arena, n, jb0, jb1);
        ++calls;
        if (sc.status != kStatusOk || !(sc.score < min_score)) break;
        min_score = sc.score;
        if (lane < m) sc.log_sp[lane] = sc.trial[lane];
        __syncwarp();
      }
      if (sc.status != kStatusOk) break;
    }
  }
  // terminal Newton polish from the selected point
  if (sc.status == kStatusOk) {
    __syncwarp();
    if (lane < m) sc.trial[lane] = sc.log_sp[lane];
    __syncwarp();
    warp_core(arena, n, jb0, jb1);
    for (int ps = 0; ps < kPolishSteps && sc.status == kStatusOk; ++ps) {
      warp_derivatives(arena, n, jrow);
      if (lane == 0) sc.ctl = polish_step(m, &sc);
      __syncwarp();
      const int act = sc.ctl;
      __syncwarp();
      if (act == 0) break;
      if (lane < m) sc.trial[lane] = sc.log_sp[lane];
      __syncwarp();
      warp_core(arena, n, jb0, jb1);
      ++calls;
      if (act == 2) break;
    }
  }
  // final fit at the selected point (the last core call may be a rejected probe)
  if (sc.status == kStatusOk) {
    __syncwarp();
    if (lane < m) sc.trial[lane] = sc.log_sp[lane];
    __syncwarp();
    warp_core(arena, n, jb0, jb1);
  }
  const double* wg = sm + L::WG;
  double* r = residuals + static_cast<int64_t>(n) * job.out;
  const bool ok = sc.status == kStatusOk;
  for (int i = lane; i < n; i += 32) {
    double f = 0.0;
    if (ok)
      for (int c = 0; c < q; ++c) f += Q[i + static_cast<int64_t>(n) * c] * wg[c];
    r[i] = ok ? y[i] - f : NAN;
  }
  if (lane == 0)
    store_result(results + t, sc.log_sp, m, sc.score, sc.edf, sc.rss, sc.status, it, calls,
                 sc.dropped > 0 ? kFitRankTruncated : 0);
}

// ------------------------------------------------------ speculative continuation
//
// fit_multi_spec_kernel: the fits that fit_multi_warp_kernel deferred (more
// than defer_calls evaluations), one per CTA of kSpecWarps warps, each warp
// with its own slot.  Within a Newton iteration magic's trial steps are fixed
// in advance -- the Newton step halved for tries 1-3, then (unless already
// steepest) the steepest-descent step halved, the step zero at try 25 -- and
// a trial is accepted on its own score, so the warps evaluate kSpecWarps
// consecutive trials at once and the first accepted one in sequence order is
// taken: the same point, score and derivatives as the sequential search.  The
// boundary probes are speculated the same way; the terminal polish and the
// final fit run on warp 0.
constexpr int kSpecWarps = 6;
constexpr int kSpecCtas = 148 * (6 / kSpecWarps);  // as many CTAs as the SMs' shared memory holds

struct SpecShared {
  double score[kSpecWarps];
  int status[kSpecWarps];
  int dec;                    // decision broadcast: accepted / failed trial
  int dec_warp;
  double log_sp[kWarpM];      // state after the accepted trial
  double newton[kWarpM];
  double steep[kWarpM];
  double gradient[kWarpM];
  double min_score;
  double score_red;
  int steepest;
  int converged;
  int fail;
};

// warp_derivatives of the trial warp ``aw`` accepted, with the q-length dot
// products -- the entries of WT = W T and of C = T'T and D = (WT)'(WT) --
// spread over all kSpecWarps warps of the CTA; every sum whose order matters
// (the sum of squares of WT, the block sums over the columns b) stays on warp
// aw in warp_derivatives' order, so the results are the same bits.  C and D
// go to the X regions of two other warps (stride 33: no bank conflicts),
// which hold nothing between trials.  Called by every warp of the CTA.
__device__ __noinline__ void spec_derivatives(const double* __restrict__ arena, int n, int jrow, int aw) {
  using L = WarpLayout;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sm = s_warp_dyn + aw * kWarpSlotDoubles;
  const WarpDesign& des = *reinterpret_cast<const WarpDesign*>(sm + L::TOTAL + kWarpScalarDoubles);
  const WarpScalars& sc = *reinterpret_cast<const WarpScalars*>(sm + L::TOTAL);
  const int q = des.q;
  double* X = sm + L::X;
  const double* Y = sm + L::Y;
  const double* Z = sm + L::Z;
  double* Cb = s_warp_dyn + ((aw + 1) % kSpecWarps) * kWarpSlotDoubles + L::X;
  double* Db = s_warp_dyn + ((aw + 2) % kSpecWarps) * kWarpSlotDoubles + L::X;
  if (warp == aw) deriv_setup(sm, arena, jrow);
  __syncthreads();
  for (int i = warp; i < q; i += kSpecWarps)
    X[kWarpR * i + lane] = warp_dot(Y + packed_row(i, 0) + i, Z + lane + kWarpR * i, kWarpR, q - i);
  __syncthreads();
  for (int b = warp; b < kWarpR; b += kSpecWarps) {
    double c = 0.0, d = 0.0;
    for (int i = 0; i < q; ++i) {
      c = fma(Z[kWarpR * i + lane], Z[kWarpR * i + b], c);
      d = fma(X[kWarpR * i + lane], X[kWarpR * i + b], d);
    }
    Cb[33 * lane + b] = c;
    Db[33 * lane + b] = d;
  }
  __syncthreads();
  if (warp == aw) {
    double dd = 0.0;
    for (int i = 0; i < q; ++i) {
      const double s = X[kWarpR * i + lane];
      dd = fma(s, s, dd);
    }
    double p[kWarpM][4];
#pragma unroll
    for (int bj = 0; bj < kWarpM; ++bj) p[bj][0] = p[bj][1] = p[bj][2] = p[bj][3] = 0.0;
    for (int b = 0; b < kWarpR; ++b) block_term(b, Cb[33 * lane + b], Db[33 * lane + b], sm + L::AV, sm + L::BV, sc, p);
    deriv_finish(sm, n, p, dd);
  }
}

__global__ void __launch_bounds__(32 * kSpecWarps) fit_multi_spec_kernel(
    const DesignDev* __restrict__ designs, const double* __restrict__ arena, const double* __restrict__ data, int n,
    const FitJob* __restrict__ jobs, const int* __restrict__ defer_list, const int* __restrict__ defer_count,
    const FitState* __restrict__ states, double* __restrict__ residuals, FitResult* __restrict__ results) {
  using L = WarpLayout;
  __shared__ SpecShared ss;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = *defer_count;
  const int max_half = 25;
  for (int di = blockIdx.x; di < total; di += gridDim.x) {
    const int t = defer_list[di];
    const FitJob job = jobs[t];
    const double* y = data + static_cast<int64_t>(n) * job.column;
    int jb0 = -1, jb1 = -1, jrow = -1;
    warp_fit_setup(designs + job.design, arena, y, n, &jb0, &jb1, &jrow);
    WarpScalars& sc = warp_scalars();
    const WarpDesign& des = warp_design();
    const int m = des.m, q = des.q;
    const FitState& st = states[t];
    if (lane < m) {
      sc.log_sp[lane] = st.log_sp[lane];
      sc.newton[lane] = st.newton[lane];
      sc.steep[lane] = st.steep[lane];
      sc.gradient[lane] = st.gradient[lane];
      for (int j = 0; j < m; ++j) sc.hess_c[lane + WarpScalars::kLd * j] = st.hess[lane + kWarpM * j];
    }
    double min_score = st.min_score;
    int calls = st.calls;
    bool steepest = st.steepest != 0;
    bool converged = false;
    int status = kStatusOk;
    int it = st.it;
    __syncwarp();
    for (; it <= kMaxIterations && status == kStatusOk; ++it) {
      // trial tt (1-based) of this iteration: tt <= 3 Newton (unless
      // steepest), then steepest descent, halved at every rejection; zero at 25
      const bool s0 = steepest;
      int accepted = 0, failed = 0, tries = 0;
      for (int base = 1; base <= max_half && !accepted && !failed; base += kSpecWarps) {
        const int tt = base + warp;
        if (tt <= max_half) {
          if (lane < m) {
            double stp;
            if (tt == max_half) stp = 0.0;
            else if (!s0 && tt <= 3) stp = ldexp(sc.newton[lane], -(tt - 1));
            else if (!s0) stp = ldexp(sc.steep[lane], -(tt - 4));
            else stp = ldexp(sc.steep[lane], -(tt - 1));
            sc.trial[lane] = sc.log_sp[lane] + stp;
          }
          __syncwarp();
          warp_core(arena, n, jb0, jb1);
          if (lane == 0) {
            ss.score[warp] = sc.score;
            ss.status[warp] = sc.status;
          }
        }
        __syncthreads();
        for (int w = 0; w < kSpecWarps && base + w <= max_half; ++w) {
          tries = base + w;
          if (ss.status[w] != kStatusOk) {
            failed = ss.status[w];
            break;
          }
          if (ss.score[w] < min_score) {
            accepted = w + 1;  // warp index + 1
            break;
          }
        }
        __syncthreads();
      }
      calls += tries;
      if (failed) {
        status = failed;
        break;
      }
      if (accepted) {
        const int aw = accepted - 1;
        if (warp == aw) {
          if (lane == 0) {
            ss.score_red = min_score - sc.score;
            ss.min_score = sc.score;
          }
          if (lane < m) sc.log_sp[lane] = sc.trial[lane];
          __syncwarp();
        }
        spec_derivatives(arena, n, jrow, aw);  // every warp of the CTA takes part
        if (warp == aw) {
          double g2 = 0.0;
          for (int r = 0; r < m; ++r) g2 += sc.gradient[r] * sc.gradient[r];  // the previous gradient
          bool conv = false;
          if (it > 3) {
            const double ms = ss.min_score;
            conv = ss.score_red <= kConvTol * (1.0 + ms) && sqrt(g2) <= pow(kConvTol, 1.0 / 3.0) * (1.0 + fabs(ms));
          }
          if (lane == 0) {
            for (int r = 0; r < m; ++r) sc.gradient[r] = sc.grad_c[r];
            bool stp = false;
            newton_from_hessian(m, &sc, &stp);
            ss.steepest = stp ? 1 : 0;
            ss.converged = conv ? 1 : 0;
            ss.fail = sc.status;
            for (int r = 0; r < m; ++r) {
              ss.log_sp[r] = sc.log_sp[r];
              ss.newton[r] = sc.newton[r];
              ss.steep[r] = sc.steep[r];
              ss.gradient[r] = sc.gradient[r];
            }
          }
          __syncwarp();
        }
        __syncthreads();
        // every warp takes the accepted state
        if (lane < m) {
          sc.log_sp[lane] = ss.log_sp[lane];
          sc.newton[lane] = ss.newton[lane];
          sc.steep[lane] = ss.steep[lane];
          sc.gradient[lane] = ss.gradient[lane];
        }
        __syncwarp();
        min_score = ss.min_score;
        steepest = ss.steepest != 0;
        converged = ss.converged != 0;
        if (ss.fail != kStatusOk) status = ss.fail;
        __syncthreads();
      } else {
        // no decrease in 25 tries: converged; the Newton direction is unchanged
        if (it > 3) converged = true;
      }
      if (converged || status != kStatusOk) break;
    }
    if (status == kStatusOk && !converged) status = kStatusNotConverged;
    // boundary probes: +-2 up to five times per coordinate, kSpecWarps at once
    if (status == kStatusOk) {
      for (int c = 0; c < m && status == kStatusOk; ++c) {
        const double direction = sc.gradient[c] < 0.0 ? 1.0 : -1.0;
        int taken = 0;
        bool stop = false;
        for (int base = 1; base <= 5 && !stop; base += kSpecWarps) {
          const int k = base + warp;  // probe k moves coordinate c by 2 k, as k successive +-2 steps
          if (k <= 5) {
            if (lane < m) {
              double v = sc.log_sp[lane];
              if (lane == c)
                for (int u = 0; u < k; ++u) v = v + direction * 2.0;
              sc.trial[lane] = v;
            }
            __syncwarp();
            warp_core(arena, n, jb0, jb1);
            if (lane == 0) {
              ss.score[warp] = sc.score;
              ss.status[warp] = sc.status;
            }
          }
          __syncthreads();
          double best = min_score;
          for (int w = 0; w < kSpecWarps && base + w <= 5; ++w) {
            ++calls;
            if (ss.status[w] != kStatusOk) {
              status = ss.status[w];
              stop = true;
              break;
            }
            if (!(ss.score[w] < best)) {
              stop = true;
              break;
            }
            best = ss.score[w];
            taken = base + w;
          }
          min_score = best;
          __syncthreads();
        }
        if (lane == c)
          for (int u = 0; u < taken; ++u) sc.log_sp[c] = sc.log_sp[c] + direction * 2.0;
        __syncwarp();
      }
    }
    // terminal polish and the final fit on warp 0
    if (warp == 0) {
      if (status == kStatusOk) {
        if (lane == 0) sc.status = kStatusOk;
        if (lane < m) sc.trial[lane] = sc.log_sp[lane];
        __syncwarp();
        warp_core(arena, n, jb0, jb1);
        for (int ps = 0; ps < kPolishSteps && sc.status == kStatusOk; ++ps) {
          warp_derivatives(arena, n, jrow);
          if (lane == 0) sc.ctl = polish_step(m, &sc);
          __syncwarp();
          const int act = sc.ctl;
          __syncwarp();
          if (act == 0) break;
          if (lane < m) sc.trial[lane] = sc.log_sp[lane];
          __syncwarp();
          warp_core(arena, n, jb0, jb1);
          ++calls;
          if (act == 2) break;
        }
        if (sc.status == kStatusOk) {
          __syncwarp();
          if (lane < m) sc.trial[lane] = sc.log_sp[lane];
          __syncwarp();
          warp_core(arena, n, jb0, jb1);
        }
        status = sc.status;
      }
      const double* Q = arena + des.basis;
      const double* wg = warp_slot() + L::WG;
      double* r = residuals + static_cast<int64_t>(n) * job.out;
      const bool ok = status == kStatusOk;
      for (int i = lane; i < n; i += 32) {
        double f = 0.0;
        if (ok)
          for (int c = 0; c < q; ++c) f += Q[i + static_cast<int64_t>(n) * c] * wg[c];
        r[i] = ok ? y[i] - f : NAN;
      }
      if (lane == 0)
        store_result(results + t, sc.log_sp, m, sc.score, sc.edf, sc.rss, status, it, calls,
                     sc.dropped > 0 ? kFitRankTruncated : 0);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------ GCV adjoint
//
// Score V, gradient, exact Hessian and Gauss-Newton Hessian of V in
// rho = log(lambda) at caller-given points (one warp or one CTA per point),
// for one additive design and one response column.  The same evaluation and
// derivative routines as the fit kernels; no optimiser.  Outputs per point:
// score[pt], grad[pt*m + j], gn / hess[(pt*m + i)*m + j], status[pt].

__global__ void __launch_bounds__(32) gcv_adjoint_warp_kernel(const DesignDev* __restrict__ designs, int design,
                                                              const double* __restrict__ arena,
                                                              const double* __restrict__ y, int n,
                                                              const double* __restrict__ rho, int count,
                                                              double* __restrict__ score, double* __restrict__ grad,
                                                              double* __restrict__ gn, double* __restrict__ hess,
                                                              int* __restrict__ status) {
  WarpScalars& sc = warp_scalars();
  const WarpDesign& des = warp_design();
  const int pt = blockIdx.x;
  if (pt >= count) return;
  const int lane = threadIdx.x & 31;
  int jb0 = -1, jb1 = -1, jrow = -1;
  warp_fit_setup(designs + design, arena, y, n, &jb0, &jb1, &jrow);
  const int m = des.m;
  if (lane < m) {
    sc.trial[lane] = rho[static_cast<int64_t>(pt) * m + lane];
    sc.log_sp[lane] = sc.trial[lane];
  }
  __syncwarp();
  warp_core(arena, n, jb0, jb1);
  if (sc.status == kStatusOk) warp_derivatives(arena, n, jrow);
  if (lane == 0) {
    score[pt] = sc.score;
    status[pt] = sc.status;
    for (int i = 0; i < m; ++i) {
      grad[static_cast<int64_t>(pt) * m + i] = sc.grad_c[i];
      for (int j = 0; j < m; ++j) {
        gn[(static_cast<int64_t>(pt) * m + i) * m + j] = sc.gn_c[i + WarpScalars::kLd * j];
        hess[(static_cast<int64_t>(pt) * m + i) * m + j] = sc.hess_c[i + WarpScalars::kLd * j];
      }
    }
  }
}

template <int QMAX, int RMAX>
__global__ void __launch_bounds__(kMultiThreads, 1) gcv_adjoint_kernel(
    const DesignDev* __restrict__ designs, int design, const double* __restrict__ arena, const double* __restrict__ y,
    int n, const double* __restrict__ rho, int count, double* __restrict__ score, double* __restrict__ grad,
    double* __restrict__ gn, double* __restrict__ hess, int* __restrict__ status, double* __restrict__ workspace) {
  using L = MultiLayout<QMAX, RMAX>;
  extern __shared__ double smem_dyn[];
  double* sm = workspace ? workspace + static_cast<int64_t>(blockIdx.x) * L::TOTAL : smem_dyn;
  __shared__ MultiScalars sc;
  const int pt = blockIdx.x;
  if (pt >= count) return;
  const DesignDev& des = designs[design];
  const int tid = threadIdx.x;
  const int m = des.m;
  multi_fit_setup<QMAX, RMAX, MultiScalars, DesignDev>(des, arena, y, n, sm, sc);
  if (tid < m) {
    sc.trial[tid] = rho[static_cast<int64_t>(pt) * m + tid];
    sc.log_sp[tid] = sc.trial[tid];
  }
  __syncthreads();
  multi_core<QMAX, RMAX>(des, arena, n, sm, &sc);
  if (sc.status == kStatusOk) multi_derivatives<QMAX, RMAX>(des, arena, n, sm, &sc);
  if (tid == 0) {
    score[pt] = sc.score;
    status[pt] = sc.status;
    for (int i = 0; i < m; ++i) {
      grad[static_cast<int64_t>(pt) * m + i] = sc.grad_c[i];
      for (int j = 0; j < m; ++j) {
        gn[(static_cast<int64_t>(pt) * m + i) * m + j] = sc.gn_c[i + MultiScalars::kLd * j];
        hess[(static_cast<int64_t>(pt) * m + i) * m + j] = sc.hess_c[i + MultiScalars::kLd * j];
      }
    }
  }
}

size_t multi_smem_bytes(int qmax_class) {
  if (qmax_class == 0) return kWarpSlotBytes;
  if (qmax_class == 1) return sizeof(double) * MultiLayout<76, 64>::TOTAL;
  return 0;  // class 2 works in global memory
}

// CTAs of the wide class's persistent launch (one per SM at most).
int wide_ctas(int count) { return count < 148 ? count : 148; }

size_t multi_workspace_doubles(int qmax_class, int count) {
  if (qmax_class == 2) return static_cast<size_t>(MultiLayout<112, 96>::TOTAL) * static_cast<size_t>(count);
  if (qmax_class == 3) return static_cast<size_t>(kWideSlotDoubles) * static_cast<size_t>(wide_ctas(count));
  return 0;
}

cudaError_t configure_fit_kernels() {
  cudaError_t e = cudaFuncSetAttribute(fit_multi_warp_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fit_multi_spec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kSpecWarps * kWarpSlotBytes));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fit_multi_kernel<76, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(multi_smem_bytes(1)));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(gcv_adjoint_kernel<76, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(multi_smem_bytes(1)));
}

cudaError_t launch_gcv_adjoint(int qmax_class, const DesignDev* designs, int design, const double* arena,
                               const double* y, int n, const double* rho, int count, double* score, double* grad,
                               double* gn, double* hess, int* status, cudaStream_t stream, double* workspace) {
  if (count <= 0) return cudaSuccess;
  if (qmax_class == 0) {
    gcv_adjoint_warp_kernel<<<count, 32, kWarpSlotBytes, stream>>>(designs, design, arena, y, n, rho, count, score,
                                                                   grad, gn, hess, status);
  } else if (qmax_class == 1) {
    gcv_adjoint_kernel<76, 64><<<count, kMultiThreads, multi_smem_bytes(1), stream>>>(
        designs, design, arena, y, n, rho, count, score, grad, gn, hess, status, nullptr);
  } else {
    if (!workspace) return cudaErrorInvalidValue;
    gcv_adjoint_kernel<112, 96><<<count, kMultiThreads, 0, stream>>>(designs, design, arena, y, n, rho, count, score,
                                                                      grad, gn, hess, status, workspace);
  }
  return cudaGetLastError();
}

cudaError_t launch_fit_single(const DesignDev* designs, const double* arena, const double* data, int n,
                              const FitJob* jobs, int count, double* residuals, FitResult* results,
                              cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const int warps = 8;
  dim3 grid((count + warps - 1) / warps);
  fit_single_kernel<<<grid, warps * 32, 0, stream>>>(designs, arena, data, n, jobs, count, residuals, results);
  return cudaGetLastError();
}

cudaError_t launch_fit_multi(int qmax_class, const DesignDev* designs, const double* arena, const double* data,
                             int n, const FitJob* jobs, const int* job_index, int count, double* residuals,
                             FitResult* results, cudaStream_t stream, int selection, double* workspace,
                             FitState* states, int* defer_list, int* defer_count, cudaEvent_t after_warp,
                             int defer_calls, double* wide_log_sp) {
  if (count <= 0) return cudaSuccess;
  if (qmax_class == 0) {
    // fits still searching after defer_calls evaluations continue in the
    // speculative kernel (magic selection, with the deferral buffers given)
    const bool defer = states && defer_list && defer_count && selection == FKPC_SELECT_MAGIC && defer_calls > 0;
    if (defer) {
      cudaError_t e = cudaMemsetAsync(defer_count, 0, sizeof(int), stream);
      if (e != cudaSuccess) return e;
    }
    fit_multi_warp_kernel<<<count, 32, kWarpSlotBytes, stream>>>(designs, arena, data, n, jobs, job_index, count,
                                                                 residuals, results, selection,
                                                                 defer ? defer_calls : 0, states, defer_list,
                                                                 defer_count);
    if (after_warp) {
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaEventRecord(after_warp, stream);
      if (e != cudaSuccess) return e;
    }
    if (defer) {
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      const int ctas = count < kSpecCtas ? count : kSpecCtas;
      fit_multi_spec_kernel<<<ctas, 32 * kSpecWarps, kSpecWarps * kWarpSlotBytes, stream>>>(
          designs, arena, data, n, jobs, defer_list, defer_count, states, residuals, results);
    }
  } else if (qmax_class == 1) {
    fit_multi_kernel<76, 64><<<count, kMultiThreads, multi_smem_bytes(1), stream>>>(
        designs, arena, data, n, jobs, job_index, count, residuals, results, selection, nullptr);
  } else if (qmax_class == 2) {
    if (!workspace) return cudaErrorInvalidValue;
    fit_multi_kernel<112, 96><<<count, kMultiThreads, 0, stream>>>(designs, arena, data, n, jobs, job_index, count,
                                                                    residuals, results, selection, workspace);
  } else {
    if (!workspace || !wide_log_sp) return cudaErrorInvalidValue;
    fit_multi_wide_kernel<<<wide_ctas(count), kWideThreads, 0, stream>>>(designs, arena, data, n, jobs, job_index,
                                                                        count, residuals, results, selection,
                                                                        workspace, wide_log_sp);
  }
  return cudaGetLastError();
}

}  // namespace fkpc
