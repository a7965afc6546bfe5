// Independence statistics and p-values on the GPU (FP64).
//
// dCov (fastkpc/src/cuda/full_cuda_ci_vertical.cu:485-769 restated without
// any n x n buffer): per component the row-centring constants
// c_i = mean_j |r_i - r_j| - grand/2 (so A_ij = |r_i - r_j| - c_i - c_j), the
// distance total and sum A^2; per pair sum A_ij B_ij over the upper triangle
// with both residual vectors and their constants staged in shared memory,
// then nV2, the gamma moments and the upper tail in the same CTA.
//
// Legacy low-rank dCov for the guard band (kpcalg/R/dcovgamma.R:51-100;
// fastkpc/src/cuda/full_cuda_ci_vertical.cu:771-967): the num_col eigenpairs
// of largest |value| of the raw distance matrix by Lanczos with full
// re-orthogonalisation (distance entries recomputed on the fly), Ritz
// vectors from inverse iteration on the tridiagonal, centred.
//
// HSIC (kpcalg/R/hsicgamma.R:52-99; fastkpc/src/cuda/full_cuda_ci_method_batch.cu:445-789):
// kernlab-style incomplete Cholesky of the RBF Gram per component, pair
// statistic |Gx' Gy|_F^2 / n^2, gamma moments, p = 1 - (1 - Q).
// Permutation forms (fastkpc/src/cuda/full_cuda_ci_method_batch.cu:341-443,
// :791-908): p = (1 + #{T_pi >= T}) / (R + 1).
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>

#include "device.h"
#include "kernels.h"

namespace fkpc {

namespace {

constexpr int kStatThreads = 256;
constexpr double kIncholTol = 1e-3;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Work item b of a launch: b itself, or the b-th entry of a device index list.
__device__ __forceinline__ int work_item(const WorkList& wl, int b, int count) {
  if (!wl.idx) return b < count ? b : -1;
  if (b >= *wl.count || b >= count) return -1;
  const int v = wl.idx[b];
  return (v >= 0 && v < count) ? v : -1;  // an entry outside the launch's range is never used
}

__device__ double block_sum256(double v, double* red) {
  v = warp_sum(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

// ---------------------------------------------------------------- gamma tail
// Q(a, x) = Gamma(a, x) / Gamma(a), the upper tail of the gamma law the
// dCov / HSIC moments define.  Written from two published representations:
//
//  * x < a + 1: the lower function by its power series (DLMF 8.7.1 / 8.11.4),
//      P(a, x) = x^a e^-x / Gamma(a + 1) * sum_k x^k / ((a + 1) ... (a + k)),
//    and Q = 1 - P (P is at most about 0.6 here, so Q keeps its absolute bits);
//  * otherwise: Legendre's continued fraction for Gamma(a, x) (DLMF 8.9.2),
//      e^x x^-a Gamma(a, x) = 1 / (x + 1 - a) * 1 / (1 + al_1 / (1 + al_2 / (1 + ...))),
//      al_k = k (a - k) / ((x + 2k - 1 - a)(x + 2k + 1 - a)),
//    summed as a series by the forward recurrence of W. Gautschi (ACM TOMS 5
//    (1979) 466-481, section 4): t_0 = 1, r_0 = 0,
//      r_k = -al_k (1 + r_{k-1}) / (1 + al_k (1 + r_{k-1})),  t_k = r_k t_{k-1}.
//    For x >= a + 1 every |al_k| with k > a is below 1/4, so the denominators
//    stay above 1/2: the recurrence needs no underflow guard.
//
// The common factor x^a e^-x / Gamma(a) is formed without cancellation for
// a >= 10 through Stirling's series (Gamma(a) = sqrt(2 pi / a) (a / e)^a
// e^{st(a)}, st(a) = sum_k B_2k / (2k (2k - 1) a^(2k-1))):
//      x^a e^-x / Gamma(a) = sqrt(a / (2 pi)) exp(-a phi((x - a) / a) - st(a)),
//      phi(t) = t - log(1 + t) >= 0,
// with phi near 0 from the atanh series of log(1 + t) in u = t / (2 + t).
// Both sums stop once a term falls below 2^-56 of the running sum; after
// kGammaMaxTerms terms *ok stays 0.
constexpr int kGammaMaxTerms = 20000;

// t - log1p(t), accurate near t = 0
__device__ double gamma_phi(double t) {
  if (fabs(t) < 0.5) {
    const double u = t / (2.0 + t), u2 = u * u;
    double s = 0.0;  // 1/3 + u^2/5 + u^4/7 + ... (Horner, from the tail)
    for (int k = 41; k >= 3; k -= 2) s = fma(s, u2, 1.0 / k);
    return 2.0 * u2 / (1.0 - u) - 2.0 * u * u2 * s;
  }
  return t - log1p(t);
}

// log(Gamma(a)) - ((a - 1/2) log a - a + log(2 pi) / 2) for a >= 10
__device__ double gamma_stirling_tail(double a) {
  const double ia2 = 1.0 / (a * a);
  double s = 1.0 / 156.0;
  s = fma(s, ia2, -691.0 / 360360.0);
  s = fma(s, ia2, 1.0 / 1188.0);
  s = fma(s, ia2, -1.0 / 1680.0);
  s = fma(s, ia2, 1.0 / 1260.0);
  s = fma(s, ia2, -1.0 / 360.0);
  s = fma(s, ia2, 1.0 / 12.0);
  return s / a;
}

// x^a e^-x / Gamma(a), x > 0
__device__ double gamma_kernel_factor(double a, double x) {
  if (a < 10.0) return exp(a * log(x) - x - lgamma(a));
  return sqrt(a * 0.15915494309189533577 /* 1 / (2 pi) */) * exp(-a * gamma_phi((x - a) / a) - gamma_stirling_tail(a));
}

__device__ double gamma_q(double a, double x, int* ok) {
  *ok = 0;
  if (!(a > 0.0) || !(x >= 0.0) || !isfinite(a) || !isfinite(x)) return NAN;
  *ok = 1;
  if (x == 0.0) return 1.0;
  const double eps = 0x1p-56;
  if (x < a + 1.0) {
    double sum = 1.0, term = 1.0;
    for (int k = 1; k <= kGammaMaxTerms; ++k) {
      term *= x / (a + k);
      sum += term;
      if (term <= eps * sum) return fmin(1.0, fmax(0.0, 1.0 - gamma_kernel_factor(a, x) / a * sum));
    }
  } else {
    double sum = 1.0, t = 1.0, r = 0.0;
    for (int k = 1; k <= kGammaMaxTerms; ++k) {
      const double al = k * (a - k) / ((x + (2 * k - 1) - a) * (x + (2 * k + 1) - a));
      const double w = al * (1.0 + r);
      r = -w / (1.0 + w);
      t *= r;
      sum += t;
      if (fabs(t) <= eps * fabs(sum)) return fmin(1.0, gamma_kernel_factor(a, x) / (x + 1.0 - a) * sum);
    }
  }
  *ok = 0;
  return NAN;
}

__device__ double var_factor(double n) {
  return 2.0 * (n - 4.0) * (n - 5.0) / n / (n - 1.0) / (n - 2.0) / (n - 3.0);
}

// statistic, moments -> record with the gamma upper tail
__device__ void gamma_record(double stat, double mean, double var, bool hsic, RecordDev* out) {
  out->statistic = stat;
  out->mean = mean;
  out->variance = var;
  out->flags = 0;
  if (!isfinite(stat) || !isfinite(mean) || !isfinite(var) || !(mean > 0.0) || !(var > 0.0)) {
    out->status = kStatusNumeric;
    out->p_value = NAN;
    out->p_exact = NAN;
    return;
  }
  const double shape = mean * mean / var;
  const double scale = var / mean;
  int ok = 0;
  double p = gamma_q(shape, fmax(0.0, stat / scale), &ok);
  if (!ok || !isfinite(p)) {
    out->status = kStatusNotConverged;
    out->p_value = NAN;
    out->p_exact = NAN;
    return;
  }
  if (hsic) p = 1.0 - (1.0 - fmin(1.0, fmax(0.0, p)));
  out->status = kStatusOk;
  out->p_value = p;
  out->p_exact = p;
}

}  // namespace

// ------------------------------------------------------------------ dCov

__global__ void __launch_bounds__(kStatThreads) dcov_component_kernel(const double* __restrict__ residuals, int n,
                                                                       const int* __restrict__ comp_cols, int count,
                                                                       double* __restrict__ centre,
                                                                       DcovComponent* __restrict__ comps,
                                                                       WorkList wl) {
  extern __shared__ double sm[];
  __shared__ double red[kStatThreads / 32];
  const int comp = work_item(wl, blockIdx.x, count);
  if (comp < 0) return;
  double* r = sm;
  double* c = sm + n;
  const double* src = residuals + static_cast<int64_t>(n) * comp_cols[comp];
  for (int i = threadIdx.x; i < n; i += blockDim.x) r[i] = src[i];
  __syncthreads();
  double part = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double ri = r[i];
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += fabs(ri - r[j]);
    c[i] = s;
    part += s;
  }
  const double total = block_sum256(part, red);
  const double nd = static_cast<double>(n);
  const double half_grand = 0.5 * total / (nd * nd);
  for (int i = threadIdx.x; i < n; i += blockDim.x) c[i] = c[i] / nd - half_grand;
  __syncthreads();
  // sum A^2 over the upper triangle (rows i and n-1-i per thread), plus diagonal
  double acc = 0.0;
  const int half = (n + 1) / 2;
  for (int t = threadIdx.x; t < half; t += blockDim.x) {
    const int a = t, b = n - 1 - t;
    {
      const double ra = r[a], ca = c[a];
      for (int j = a + 1; j < n; ++j) {
        const double v = fabs(ra - r[j]) - ca - c[j];
        acc += v * v;
      }
    }
    if (b != a) {
      const double rb = r[b], cb = c[b];
      for (int j = b + 1; j < n; ++j) {
        const double v = fabs(rb - r[j]) - cb - c[j];
        acc += v * v;
      }
    }
  }
  double diag = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) diag += 4.0 * c[i] * c[i];
  const double self = 2.0 * block_sum256(acc, red) + block_sum256(diag, red);
  double* cout = centre + static_cast<int64_t>(n) * comp;
  for (int i = threadIdx.x; i < n; i += blockDim.x) cout[i] = c[i];
  if (threadIdx.x == 0) {
    comps[comp].total = total;
    comps[comp].self = self;
  }
}

__global__ void __launch_bounds__(kStatThreads) dcov_pair_kernel(const double* __restrict__ residuals, int n,
                                                                  const int* __restrict__ comp_cols,
                                                                  const double* __restrict__ centre,
                                                                  const DcovComponent* __restrict__ comps,
                                                                  const PairJob* __restrict__ pairs, int count,
                                                                  RecordDev* __restrict__ records, WorkList wl) {
  extern __shared__ double sm[];
  __shared__ double red[kStatThreads / 32];
  const int t = work_item(wl, blockIdx.x, count);
  if (t < 0) return;
  const PairJob job = pairs[t];
  double* x = sm;
  double* cx = sm + n;
  double* y = sm + 2 * n;
  double* cy = sm + 3 * n;
  const double* xs = residuals + static_cast<int64_t>(n) * comp_cols[job.left];
  const double* ys = residuals + static_cast<int64_t>(n) * comp_cols[job.right];
  const double* cxs = centre + static_cast<int64_t>(n) * job.left;
  const double* cys = centre + static_cast<int64_t>(n) * job.right;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    x[i] = xs[i];
    y[i] = ys[i];
    cx[i] = cxs[i];
    cy[i] = cys[i];
  }
  __syncthreads();
  double acc = 0.0;
  const int half = (n + 1) / 2;
  for (int tt = threadIdx.x; tt < half; tt += blockDim.x) {
    const int a = tt, b = n - 1 - tt;
    {
      const double xa = x[a], ya = y[a], ca = cx[a], da = cy[a];
      for (int j = a + 1; j < n; ++j) {
        const double u = fabs(xa - x[j]) - ca - cx[j];
        const double v = fabs(ya - y[j]) - da - cy[j];
        acc = fma(u, v, acc);
      }
    }
    if (b != a) {
      const double xb = x[b], yb = y[b], cb = cx[b], db = cy[b];
      for (int j = b + 1; j < n; ++j) {
        const double u = fabs(xb - x[j]) - cb - cx[j];
        const double v = fabs(yb - y[j]) - db - cy[j];
        acc = fma(u, v, acc);
      }
    }
  }
  double diag = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) diag += 4.0 * cx[i] * cy[i];
  const double sab = 2.0 * block_sum256(acc, red) + block_sum256(diag, red);
  if (threadIdx.x == 0) {
    const double nd = static_cast<double>(n);
    const DcovComponent lx = comps[job.left], ly = comps[job.right];
    RecordDev rec;
    gamma_record(sab / nd, (lx.total / (nd * nd)) * (ly.total / (nd * nd)),
                 var_factor(nd) * lx.self * ly.self / (nd * nd), false, &rec);
    records[job.out] = rec;
  }
}

// ------------------------------------------------------ legacy low rank

namespace {

constexpr int kLanczosMax = 384;

// LU with partial pivoting of the tridiagonal (T - shift I), then solve; used
// for inverse iteration.  d, e: diagonal / off-diagonal of T (size m).
__device__ void tridiag_inverse_iteration(const double* d, const double* e, int m, double shift, double tnorm,
                                          double* x, double* l, double* u0, double* u1, double* u2, int* piv) {
  // factor
  const double small = 2.220446049250313e-16 * tnorm;
  double a = d[0] - shift;
  double b = m > 1 ? e[0] : 0.0;
  for (int i = 0; i < m; ++i) {
    const double sub = i + 1 < m ? e[i] : 0.0;        // T(i+1, i)
    const double dn = i + 1 < m ? d[i + 1] - shift : 0.0;
    const double sup2 = i + 2 < m ? e[i + 1] : 0.0;   // T(i+1, i+2)
    if (i + 1 < m && fabs(sub) > fabs(a)) {
      // swap rows i and i+1
      piv[i] = 1;
      u0[i] = sub;
      u1[i] = dn;
      u2[i] = sup2;
      const double mult = a / sub;
      l[i] = mult;
      a = b - mult * dn;
      b = -mult * sup2;
    } else {
      piv[i] = 0;
      double aa = a;
      if (fabs(aa) < small) aa = aa >= 0.0 ? small : -small;
      u0[i] = aa;
      u1[i] = b;
      u2[i] = 0.0;
      const double mult = i + 1 < m ? sub / aa : 0.0;
      l[i] = mult;
      a = dn - mult * b;
      b = sup2;
    }
  }
  for (int i = 0; i < m; ++i) {
    double piv_ = u0[i];
    if (fabs(piv_) < small) piv_ = piv_ >= 0.0 ? small : -small;
    u0[i] = 1.0 / piv_;
  }
  for (int sweep = 0; sweep < 3; ++sweep) {
    // forward (apply L and pivots)
    for (int i = 0; i + 1 < m; ++i) {
      if (piv[i]) {
        const double t = x[i];
        x[i] = x[i + 1];
        x[i + 1] = t - l[i] * x[i];
      } else {
        x[i + 1] -= l[i] * x[i];
      }
    }
    // back substitution with U (diag u0 held as reciprocals, super u1, super-2 u2)
    for (int i = m - 1; i >= 0; --i) {
      double s = x[i];
      if (i + 1 < m) s -= u1[i] * x[i + 1];
      if (i + 2 < m) s -= u2[i] * x[i + 2];
      x[i] = s * u0[i];
    }
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) nrm += x[i] * x[i];
    const double inv = 1.0 / sqrt(nrm);
    for (int i = 0; i < m; ++i) x[i] *= inv;
  }
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x: sign
// changes of the characteristic-polynomial sequence p_0 = 1,
// p_{i+1} = (d_i - x) p_i - e_{i-1}^2 p_{i-1} (Sturm), kept in range by exact
// power-of-two rescaling -- no division in the recurrence.  A zero term is
// replaced by a tiny value of the opposite sign (a negative pivot).
__device__ int sturm_count(const double* d, const double* e, int m, double x, double pivmin) {
  (void)pivmin;
  int cnt = 0;
  double pm = 0.0, pc = 1.0;
  for (int i = 0; i < m; ++i) {
    double pn = (d[i] - x) * pc - (i > 0 ? e[i - 1] * e[i - 1] * pm : 0.0);
    if (pn == 0.0) pn = -copysign(1e-300, pc) * 1e-8;
    if ((pn < 0.0) != (pc < 0.0)) ++cnt;
    pm = pc;
    pc = pn;
    const double a = fabs(pc);
    if (a > 1e150 || a < 1e-150) {
      const int ex = ilogb(a);
      pc = scalbn(pc, -ex);
      pm = scalbn(pm, -ex);
    }
  }
  return cnt;
}

// The idx-th smallest eigenvalue (0-based) of (d, e) by bisection on
// [lo, hi] until the bracket is at rounding level.
__device__ double bisect_eigenvalue(const double* d, const double* e, int m, int idx, double lo, double hi,
                                    double pivmin) {
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (hi - lo <= 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin || mid == lo || mid == hi) break;
    if (sturm_count(d, e, m, mid, pivmin) <= idx) lo = mid;
    else hi = mid;
  }
  return 0.5 * (lo + hi);
}

struct LanczosShared {
  double alpha[kLanczosMax];
  double beta[kLanczosMax];
  double td[kLanczosMax];
  double te[kLanczosMax];
  double theta[64];
  double cand[128];
  int cand_idx[128];
  int sel[64];
  double coef[kLanczosMax];
  double red[kStatThreads / 32];
  double scan[2 * (kStatThreads / 32)];
  int done;
  int steps;
  int fail;
};

// Exclusive prefix sums over the block of two per-thread values (thread
// order), with the block totals; every thread sums the warp totals in the
// same order, so the totals agree bit for bit.
__device__ void block_exscan2(double a, double c, double* scan, double* ea, double* ec, double* ta, double* tc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double ia = a, ic = c;
  for (int o = 1; o < 32; o <<= 1) {
    const double x = __shfl_up_sync(0xffffffffu, ia, o);
    const double y = __shfl_up_sync(0xffffffffu, ic, o);
    if (lane >= o) {
      ia += x;
      ic += y;
    }
  }
  __syncthreads();
  if (lane == 31) {
    scan[warp] = ia;
    scan[nw + warp] = ic;
  }
  __syncthreads();
  double oa = 0.0, oc = 0.0, sa = 0.0, sc = 0.0;
  for (int w = 0; w < nw; ++w) {
    if (w < warp) {
      oa += scan[w];
      oc += scan[nw + w];
    }
    sa += scan[w];
    sc += scan[nw + w];
  }
  *ea = oa + ia - a;
  *ec = oc + ic - c;
  *ta = sa;
  *tc = sc;
}

}  // namespace

// Grid-stride over the guarded components: CTA b handles slots b, b + grid,
// ...  guard[1] holds the slot count, slot_comps the component of each slot.
// workspace per CTA: V (n x (kLanczosMax+1)) Lanczos basis, S
// (kLanczosMax x 64) Ritz coefficient vectors, 64 x 5 x kLanczosMax
// inverse-iteration scratch (one set per thread).
__global__ void __launch_bounds__(kStatThreads, 2) legacy_eigen_kernel(const double* __restrict__ residuals, int n,
                                                                     const int* __restrict__ comp_cols,
                                                                     const int* __restrict__ guard,
                                                                     const int* __restrict__ slot_comps, int cap,
                                                                     int k, double* __restrict__ workspace,
                                                                     double* __restrict__ vals,
                                                                     double* __restrict__ vecs,
                                                                     int* __restrict__ status,
                                                                     const int* __restrict__ slot_begin) {
  extern __shared__ double sm[];
  __shared__ LanczosShared ls;
  const int slots = min(guard[1], cap);
  const int first = slot_begin ? *slot_begin : 0;
  for (int slot = first + blockIdx.x; slot < slots; slot += gridDim.x) {
  const int comp = slot_comps[slot];
  const int tid = threadIdx.x;
  const int maxit = min(n, kLanczosMax);
  double* r = sm;
  double* qv = sm + n;
  double* w = sm + 2 * n;
  int* perm = reinterpret_cast<int*>(sm + 3 * n);  // sorted position -> sample index
  const int64_t per = static_cast<int64_t>(n) * (kLanczosMax + 1) + static_cast<int64_t>(kLanczosMax) * 64 +
                      static_cast<int64_t>(64) * 5 * kLanczosMax;
  double* V = workspace + per * blockIdx.x;
  double* S = V + static_cast<int64_t>(n) * (kLanczosMax + 1);
  double* scratch = S + static_cast<int64_t>(kLanczosMax) * 64;
  const double* src = residuals + static_cast<int64_t>(n) * comp_cols[comp];
  for (int i = tid; i < n; i += blockDim.x) r[i] = src[i];
  __syncthreads();
  // Sort the residual once (rank sort on (value, index); NaN ranks as +Inf so
  // the ranks stay a permutation): the whole Lanczos runs in the sorted basis,
  // where D q is two prefix sums.  Eigenvectors are put back in sample order
  // on output.
  for (int i = tid; i < n; i += blockDim.x) {
    const double ri = isnan(r[i]) ? INFINITY : r[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double rj = isnan(r[j]) ? INFINITY : r[j];
      rank += (rj < ri || (rj == ri && j < i)) ? 1 : 0;
    }
    perm[rank] = i;
  }
  __syncthreads();
  for (int pos = tid; pos < n; pos += blockDim.x) w[pos] = r[perm[pos]];
  __syncthreads();
  for (int pos = tid; pos < n; pos += blockDim.x) r[pos] = w[pos];
  if (tid == 0) {
    ls.done = 0;
    ls.fail = 0;
    ls.steps = 0;
    unsigned long state = 1;
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) {  // start vector in sample order
      state = (state * 106UL + 1283UL) % 6075UL;
      const double v = static_cast<double>(state) / 6075.0 - 0.5;
      qv[i] = v;
      nrm += v * v;
    }
    ls.scan[0] = sqrt(nrm);
  }
  __syncthreads();
  {
    const double nrm = ls.scan[0];
    for (int pos = tid; pos < n; pos += blockDim.x) V[pos] = qv[perm[pos]] / nrm;
  }
  __syncthreads();
  double anorm = 0.0;
  for (int j = 0; j < maxit && !ls.done; ++j) {
    double* vj = V + static_cast<int64_t>(n) * j;
    for (int i = tid; i < n; i += blockDim.x) qv[i] = vj[i];
    __syncthreads();
    // w = D q, D_kl = |r_k - r_l| with r sorted: with a_k and c_k the
    // exclusive prefix sums of q and r.q, (D q)_k = r_k (2 a_k - A) + (C - 2 c_k)
    // (A, C the totals); each thread scans a contiguous chunk.
    double part = 0.0;
    {
      const int ept = (n + blockDim.x - 1) / blockDim.x;
      const int k0 = min(n, tid * ept), k1 = min(n, k0 + ept);
      double sa = 0.0, sc = 0.0;
      for (int pos = k0; pos < k1; ++pos) {
        sa += qv[pos];
        sc += r[pos] * qv[pos];
      }
      double ea, ec, ta, tc;
      block_exscan2(sa, sc, ls.scan, &ea, &ec, &ta, &tc);
      for (int pos = k0; pos < k1; ++pos) {
        const double v = r[pos] * (2.0 * ea - ta) + (tc - 2.0 * ec);
        w[pos] = v;
        part += v * qv[pos];
        ea += qv[pos];
        ec += r[pos] * qv[pos];
      }
    }
    const double alpha = block_sum256(part, ls.red);
    const double bprev = j > 0 ? ls.beta[j - 1] : 0.0;
    const double* vp = j > 0 ? V + static_cast<int64_t>(n) * (j - 1) : nullptr;
    double before = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
      double v = w[i] - alpha * qv[i];
      if (vp) v -= bprev * vp[i];
      w[i] = v;
      before += v * v;
    }
    // (the reduction's barriers also publish w)
    before = block_sum256(before, ls.red);
    // classical Gram-Schmidt against V[:, 0..j]; a second pass only when the
    // first removed more than half the norm ("twice is enough")
    double after = before;
    for (int pass = 0; pass < 2; ++pass) {
      // coefficients V(:, b)'w: each warp takes four basis vectors per pass so
      // that their L2 loads overlap
      const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
      for (int b0 = 4 * warp; b0 <= j; b0 += 4 * nwarps) {
        const double* v0 = V + static_cast<int64_t>(n) * b0;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        const bool h1 = b0 + 1 <= j, h2 = b0 + 2 <= j, h3 = b0 + 3 <= j;
#pragma unroll 4
        for (int i = lane; i < n; i += 32) {
          const double wi = w[i];
          const double x0 = v0[i];
          const double x1 = h1 ? v0[i + n] : 0.0;
          const double x2 = h2 ? v0[i + 2 * static_cast<int64_t>(n)] : 0.0;
          const double x3 = h3 ? v0[i + 3 * static_cast<int64_t>(n)] : 0.0;
          s0 += wi * x0;
          s1 += wi * x1;
          s2 += wi * x2;
          s3 += wi * x3;
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        s3 = warp_sum(s3);
        if (lane == 0) {
          ls.coef[b0] = s0;
          if (h1) ls.coef[b0 + 1] = s1;
          if (h2) ls.coef[b0 + 2] = s2;
          if (h3) ls.coef[b0 + 3] = s3;
        }
      }
      __syncthreads();
      double part2 = 0.0;
      for (int i = tid; i < n; i += blockDim.x) {
        double s0 = w[i], s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int b = 0;
        for (; b + 7 <= j; b += 8) {  // eight independent basis loads in flight
          double x[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) x[u] = V[i + static_cast<int64_t>(n) * (b + u)];
          s0 -= ls.coef[b] * x[0] + ls.coef[b + 4] * x[4];
          s1 -= ls.coef[b + 1] * x[1] + ls.coef[b + 5] * x[5];
          s2 -= ls.coef[b + 2] * x[2] + ls.coef[b + 6] * x[6];
          s3 -= ls.coef[b + 3] * x[3] + ls.coef[b + 7] * x[7];
        }
        for (; b <= j; ++b) s0 -= ls.coef[b] * V[i + static_cast<int64_t>(n) * b];
        const double s = (s0 + s1) + (s2 + s3);
        w[i] = s;
        part2 += s * s;
      }
      after = block_sum256(part2, ls.red);
      if (after > 0.25 * before) break;
      before = after;
    }
    const double beta = sqrt(after);  // |w|^2 of the last pass
    anorm = fmax(anorm, fabs(alpha) + beta + bprev);
    if (tid == 0) {
      ls.alpha[j] = alpha;
      ls.beta[j] = beta;
      ls.steps = j + 1;
    }
    const bool invariant = beta <= 1e-15 * anorm;
    const int m = j + 1;
    const int first = min(maxit, k + 40);
    const bool check = invariant || m == maxit || (m >= first && ((m - first) % 10 == 0));
    __syncthreads();
    if (check) {
      const int kk = min(k, m);
      double tnorm = 0.0, lo = INFINITY, hi = -INFINITY, bmax = 0.0;
      for (int i = 0; i < m; ++i) {
        const double bl = i > 0 ? fabs(ls.beta[i - 1]) : 0.0;
        const double br = i + 1 < m ? fabs(ls.beta[i]) : 0.0;
        lo = fmin(lo, ls.alpha[i] - bl - br);
        hi = fmax(hi, ls.alpha[i] + bl + br);
        tnorm = fmax(tnorm, fabs(ls.alpha[i]) + bl + br);
        if (i + 1 < m) bmax = fmax(bmax, ls.beta[i] * ls.beta[i]);
      }
      const double pivmin = fmax(2.2250738585072014e-308, 2.220446049250313e-16 * fmax(bmax, 1e-300));
      // candidates: the kk largest and kk smallest Ritz values (bisection, one per thread)
      if (tid < 2 * kk) {
        const int idx = tid < kk ? m - 1 - tid : tid - kk;
        if (idx >= 0 && idx < m) {
          ls.cand[tid] = bisect_eigenvalue(ls.alpha, ls.beta, m, idx, lo, hi, pivmin);
          ls.cand_idx[tid] = idx;
        } else {
          ls.cand_idx[tid] = -1;
        }
      }
      __syncthreads();
      if (tid == 0) {
        // kk largest |theta| among distinct indices (ties toward the higher
        // index).  cand[c] holds the Ritz value of rank m-1-c (descending),
        // cand[kk+c] that of rank c (ascending): merge the two ends.
        int top = 0, bot = 0;  // next candidate from each end
        for (int c = 0; c < kk; ++c) {
          const int it = m - 1 - top, ib = bot;
          bool take_top;
          if (top >= kk || it < 0) take_top = false;
          else if (bot >= kk || ib >= m || ib > it) take_top = true;
          else if (it == ib) take_top = true;  // the two ends met: one value left
          else {
            const double ft = fabs(ls.cand[top]), fb = fabs(ls.cand[kk + bot]);
            take_top = ft > fb || (ft == fb && it > ib);
          }
          if (take_top) {
            ls.sel[c] = it;
            ls.theta[c] = ls.cand[top];
            ++top;
          } else {
            ls.sel[c] = ib;
            ls.theta[c] = ls.cand[kk + bot];
            ++bot;
          }
        }
      }
      __syncthreads();
      // Ritz coefficient vectors by inverse iteration, one thread per value
      if (tid < kk) {
        double* x = S + static_cast<int64_t>(kLanczosMax) * tid;
        double* base = scratch + static_cast<int64_t>(tid) * 5 * kLanczosMax;
        for (int i = 0; i < m; ++i) x[i] = (1.0 + 0.01 * ((i * 7 + tid) % 5)) / sqrt(static_cast<double>(m));
        tridiag_inverse_iteration(ls.alpha, ls.beta, m, ls.theta[tid], tnorm, x, base, base + kLanczosMax,
                                  base + 2 * kLanczosMax, base + 3 * kLanczosMax,
                                  reinterpret_cast<int*>(base + 4 * kLanczosMax));
      }
      __syncthreads();
      if (tid == 0) {
        bool conv = m >= k;
        double tmax = 0.0;
        for (int c = 0; c < kk; ++c) tmax = fmax(tmax, fabs(ls.theta[c]));
        if (conv && !invariant) {
          for (int c = 0; c < kk; ++c) {
            const double resid = fabs(beta * S[static_cast<int64_t>(kLanczosMax) * c + (m - 1)]);
            if (resid > 1e-13 * tmax) {
              conv = false;
              break;
            }
          }
        }
        if (conv || invariant || m == maxit) ls.done = 1;
        if (ls.done && m < k) ls.fail = 1;
      }
      __syncthreads();
    }
    if (!ls.done) {
      double* vn = V + static_cast<int64_t>(n) * (j + 1);
      for (int i = tid; i < n; i += blockDim.x) vn[i] = w[i] / beta;
      __syncthreads();
    }
  }
  const int m = ls.steps;
  // order selected values descending (the order does not change any statistic)
  double* vout = vecs + static_cast<int64_t>(n) * k * slot;
  // Ritz vectors V x_c, five per pass over the basis, centred, back in sample order
  constexpr int kC = 5;
  for (int c0 = 0; c0 < k; c0 += kC) {
    double part[kC];
#pragma unroll
    for (int u = 0; u < kC; ++u) part[u] = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
      double acc[kC];
#pragma unroll
      for (int u = 0; u < kC; ++u) acc[u] = 0.0;
      int b = 0;
      for (; b + 7 < m; b += 8) {  // eight basis loads in flight
        double vb[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) vb[t] = V[i + static_cast<int64_t>(n) * (b + t)];
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
          for (int u = 0; u < kC; ++u)
            if (c0 + u < k) acc[u] += vb[t] * S[static_cast<int64_t>(kLanczosMax) * (c0 + u) + b + t];
      }
      for (; b < m; ++b) {
        const double vb = V[i + static_cast<int64_t>(n) * b];
#pragma unroll
        for (int u = 0; u < kC; ++u)
          if (c0 + u < k) acc[u] += vb * S[static_cast<int64_t>(kLanczosMax) * (c0 + u) + b];
      }
#pragma unroll
      for (int u = 0; u < kC; ++u) {
        if (c0 + u < k) vout[perm[i] + static_cast<int64_t>(n) * (c0 + u)] = acc[u];
        part[u] += acc[u];
      }
    }
#pragma unroll
    for (int u = 0; u < kC; ++u) {
      const double mean = block_sum256(part[u], ls.red) / static_cast<double>(n);
      if (c0 + u < k)
        for (int i = tid; i < n; i += blockDim.x) vout[perm[i] + static_cast<int64_t>(n) * (c0 + u)] -= mean;
    }
    __syncthreads();
  }
  if (tid < k) vals[static_cast<int64_t>(k) * slot + tid] = ls.theta[tid];
  if (tid == 0) {
    status[slot] = ls.fail ? kStatusNotConverged : kStatusOk;
    status[cap + slot] = ls.steps;
  }
  __syncthreads();
  }
}

// legacy pair: nV2 = sum l_i m_j (u_i . v_j)^2 / n; self moments per side.
// CTA t handles guarded pair guard_pairs[t] when t < guard[0].
__global__ void __launch_bounds__(kStatThreads) legacy_pair_kernel(int n, int k, const double* __restrict__ vals,
                                                                    const double* __restrict__ vecs,
                                                                    const DcovComponent* __restrict__ comps,
                                                                    const int* __restrict__ guard,
                                                                    const int* __restrict__ guard_pairs,
                                                                    const int* __restrict__ comp_slot,
                                                                    const PairJob* __restrict__ pairs, int count,
                                                                    RecordDev* __restrict__ records,
                                                                    const int* __restrict__ list_begin) {
  __shared__ double red[kStatThreads / 32];
  const int t = (list_begin ? *list_begin : 0) + blockIdx.x;
  if (t >= count || t >= guard[0]) return;
  const PairJob job = pairs[guard_pairs[t]];
  const int sx = comp_slot[job.left], sy = comp_slot[job.right];
  const double* Ux = vecs + static_cast<int64_t>(n) * k * sx;
  const double* Uy = vecs + static_cast<int64_t>(n) * k * sy;
  const double* lx = vals + static_cast<int64_t>(k) * sx;
  const double* ly = vals + static_cast<int64_t>(k) * sy;
  double cross = 0.0, selfx = 0.0, selfy = 0.0;
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    const int a = e % k, b = e / k;
    double cxy = 0.0, cxx = 0.0, cyy = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ua = Ux[i + static_cast<int64_t>(n) * a], ub = Ux[i + static_cast<int64_t>(n) * b];
      const double va = Uy[i + static_cast<int64_t>(n) * a], vb = Uy[i + static_cast<int64_t>(n) * b];
      cxy += ua * vb;
      cxx += ua * ub;
      cyy += va * vb;
    }
    cross += lx[a] * ly[b] * cxy * cxy;
    selfx += lx[a] * lx[b] * cxx * cxx;
    selfy += ly[a] * ly[b] * cyy * cyy;
  }
  cross = block_sum256(cross, red);
  selfx = block_sum256(selfx, red);
  selfy = block_sum256(selfy, red);
  if (threadIdx.x == 0) {
    const double nd = static_cast<double>(n);
    const DcovComponent cxm = comps[job.left], cym = comps[job.right];
    RecordDev rec;
    gamma_record(cross / nd, (cxm.total / (nd * nd)) * (cym.total / (nd * nd)),
                 var_factor(nd) * selfx * selfy / (nd * nd), false, &rec);
    RecordDev prev = records[job.out];
    rec.p_exact = prev.p_exact;
    rec.flags = prev.flags | FKPC_FLAG_GUARDED_DEV;
    records[job.out] = rec;
  }
}


// Guard band [lo, hi] on the exact-screen p: list the guarded pairs and give
// every component they use a low-rank slot (order of slots is irrelevant).
// guard: [0] pair count, [1] slot count, [2, 2+count) pair list,
// then comp_slot[ncomp] and slot_comps[cap].
__global__ void guard_select_kernel(const RecordDev* __restrict__ records, const PairJob* __restrict__ pairs,
                                    int count, int ncomp, int cap, double lo, double hi, int* __restrict__ guard,
                                    WorkList wl, int append, int* __restrict__ mark) {
  int* list = guard + 2;
  int* comp_slot = list + count;
  int* slot_comps = comp_slot + ncomp;
  const int items = wl.idx ? *wl.count : count;
  if (append) {
    // continue the earlier selection: record where this one starts
    if (threadIdx.x == 0) {
      mark[0] = guard[0];
      mark[1] = guard[1];
    }
    __syncthreads();
    for (int b = threadIdx.x; b < items; b += blockDim.x) {
      const int t = wl.idx ? wl.idx[b] : b;
      const PairJob job = pairs[t];
      const RecordDev rec = records[job.out];
      if (rec.status == kStatusOk && rec.p_exact >= lo && rec.p_exact <= hi) {
        const int idx = atomicAdd(guard, 1);
        list[idx] = t;
        if (comp_slot[job.left] < 0) comp_slot[job.left] = -2;
        if (comp_slot[job.right] < 0) comp_slot[job.right] = -2;
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < ncomp; c += blockDim.x) {
      if (comp_slot[c] == -2) {
        const int slot = atomicAdd(guard + 1, 1);
        if (slot < cap) {
          comp_slot[c] = slot;
          slot_comps[slot] = c;
        }
      }
    }
    return;
  }
  if (threadIdx.x == 0) {
    guard[0] = 0;
    guard[1] = 0;
  }
  for (int c = threadIdx.x; c < ncomp; c += blockDim.x) comp_slot[c] = -1;
  __syncthreads();
  for (int b = threadIdx.x; b < items; b += blockDim.x) {
    const int t = wl.idx ? wl.idx[b] : b;
    const PairJob job = pairs[t];
    const RecordDev rec = records[job.out];
    if (rec.status == kStatusOk && rec.p_exact >= lo && rec.p_exact <= hi) {
      const int idx = atomicAdd(guard, 1);
      list[idx] = t;
      comp_slot[job.left] = -2;
      comp_slot[job.right] = -2;
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncomp; c += blockDim.x) {
    if (comp_slot[c] == -2) {
      const int slot = atomicAdd(guard + 1, 1);
      if (slot < cap) {
        comp_slot[c] = slot;
        slot_comps[slot] = c;
      }
    }
  }
}

// ------------------------------------------------------------------ HSIC

__global__ void __launch_bounds__(kStatThreads) hsic_component_kernel(const double* __restrict__ residuals, int n,
                                                                       const int* __restrict__ comp_cols, int count,
                                                                       int max_rank, double sigma,
                                                                       double* __restrict__ factors,
                                                                       HsicComponent* __restrict__ comps,
                                                                       WorkList wl) {
  extern __shared__ double sm[];
  __shared__ double red[kStatThreads / 32];
  __shared__ double redv[kStatThreads / 32];
  __shared__ int redi[kStatThreads / 32];
  __shared__ double upper[64 * 64];
  __shared__ double solve[64];
  __shared__ int pivots[64];
  __shared__ double s_tau;
  __shared__ int s_pivot, s_rank, s_active;
  __shared__ double s_residue;
  const int comp = work_item(wl, blockIdx.x, count);
  if (comp < 0) return;
  const int tid = threadIdx.x;
  double* r = sm;
  double* diag = sm + n;
  double* col = sm + 2 * n;
  double* G = factors + static_cast<int64_t>(n) * max_rank * comp;
  const double* src = residuals + static_cast<int64_t>(n) * comp_cols[comp];
  for (int i = tid; i < n; i += blockDim.x) {
    r[i] = src[i];
    diag[i] = 1.0;
  }
  if (tid == 0) {
    s_residue = 1.0;
    s_pivot = 0;
    s_rank = 0;
    s_active = 1;
  }
  __syncthreads();
  while (true) {
    if (tid == 0) s_active = (s_residue > kIncholTol && s_rank < max_rank) ? 1 : 0;
    __syncthreads();
    if (!s_active) break;
    const double rp = r[s_pivot];
    for (int i = tid; i < n; i += blockDim.x) {
      const double d = r[i] - rp;
      col[i] = exp(-sigma * d * d);
    }
    __syncthreads();
    if (tid == 0) {
      const int rank = s_rank;
      double tau2 = col[s_pivot];
      for (int row = 0; row < rank; ++row) {
        double v = col[pivots[row]];
        for (int prev = 0; prev < row; ++prev) v -= upper[prev + 64 * row] * solve[prev];
        solve[row] = v / upper[row + 64 * row];
        tau2 -= solve[row] * solve[row];
        upper[row + 64 * rank] = solve[row];
      }
      if (!(tau2 > 0.0) || !isfinite(tau2)) {
        s_active = 0;
      } else {
        s_tau = sqrt(tau2);
        upper[rank + 64 * rank] = s_tau;
      }
    }
    __syncthreads();
    if (!s_active) break;
    const int rank = s_rank;
    const double tau = s_tau;
    for (int i = tid; i < n; i += blockDim.x) {
      double proj = 0.0;
      for (int prev = 0; prev < rank; ++prev) proj += G[i + static_cast<int64_t>(n) * prev] * solve[prev];
      const double upd = (col[i] - proj) / tau;
      G[i + static_cast<int64_t>(n) * rank] = upd;
      diag[i] -= upd * upd;
    }
    __syncthreads();
    // argmax of the residual diagonal, first index on ties
    double bv = -INFINITY;
    int bi = 0x7fffffff;
    for (int i = tid; i < n; i += blockDim.x) {
      if (diag[i] > bv) {
        bv = diag[i];
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) {
        bv = ov;
        bi = oi;
      }
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
      redv[warp] = bv;
      redi[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double best = redv[0];
      int besti = redi[0];
      for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2)
        if (redv[w2] > best || (redv[w2] == best && redi[w2] < besti)) {
          best = redv[w2];
          besti = redi[w2];
        }
      pivots[s_rank] = s_pivot;
      s_rank = s_rank + 1;
      s_residue = best;
      s_pivot = besti;
    }
    __syncthreads();
  }
  const int rank = s_rank;
  // off-diagonal sum of G G' from the raw factor, then centre columns
  double off = 0.0;
  double* colsum = col;  // reuse: column sums in shared memory
  for (int c = 0; c < rank; ++c) {
    double s = 0.0, s2 = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
      const double v = G[i + static_cast<int64_t>(n) * c];
      s += v;
      s2 += v * v;
    }
    s = block_sum256(s, red);
    s2 = block_sum256(s2, red);
    off += s * s - s2;
    if (tid == 0) colsum[c] = s;
    __syncthreads();
  }
  for (int c = 0; c < rank; ++c) {
    const double mean = colsum[c] / static_cast<double>(n);
    for (int i = tid; i < n; i += blockDim.x) G[i + static_cast<int64_t>(n) * c] -= mean;
  }
  __syncthreads();
  // |Gc' Gc|_F^2
  double self = 0.0;
  for (int e = tid; e < rank * rank; e += blockDim.x) {
    const int a = e % rank, b = e / rank;
    double d = 0.0;
    for (int i = 0; i < n; ++i) d += G[i + static_cast<int64_t>(n) * a] * G[i + static_cast<int64_t>(n) * b];
    self += d * d;
  }
  self = block_sum256(self, red);
  if (tid == 0) {
    comps[comp].offdiag = off;
    comps[comp].self = self;
    comps[comp].rank = rank;
    comps[comp].status = kStatusOk;
  }
}

__device__ double hsic_cross(int n, const double* Gx, int rx, const double* Gy, int ry, const int* perm,
                             double* red) {
  double acc = 0.0;
  for (int e = threadIdx.x; e < rx * ry; e += blockDim.x) {
    const int a = e % rx, b = e / rx;
    const double* ga = Gx + static_cast<int64_t>(n) * a;
    const double* gb = Gy + static_cast<int64_t>(n) * b;
    double d = 0.0;
    if (perm)
      for (int i = 0; i < n; ++i) d += ga[i] * gb[perm[i]];
    else
      for (int i = 0; i < n; ++i) d += ga[i] * gb[i];
    acc += d * d;
  }
  return block_sum256(acc, red);
}

__global__ void __launch_bounds__(kStatThreads) hsic_pair_kernel(int n, int max_rank, const double* __restrict__ factors,
                                                                  const HsicComponent* __restrict__ comps,
                                                                  const PairJob* __restrict__ pairs, int count,
                                                                  RecordDev* __restrict__ records, WorkList wl) {
  __shared__ double red[kStatThreads / 32];
  const int t = work_item(wl, blockIdx.x, count);
  if (t < 0) return;
  const PairJob job = pairs[t];
  const HsicComponent cx = comps[job.left], cy = comps[job.right];
  const double* Gx = factors + static_cast<int64_t>(n) * max_rank * job.left;
  const double* Gy = factors + static_cast<int64_t>(n) * max_rank * job.right;
  const double s = hsic_cross(n, Gx, cx.rank, Gy, cy.rank, nullptr, red);
  if (threadIdx.x == 0) {
    const double nd = static_cast<double>(n);
    const double mux = cx.offdiag / (nd * (nd - 1.0));
    const double muy = cy.offdiag / (nd * (nd - 1.0));
    RecordDev rec;
    gamma_record(s / (nd * nd), (1.0 + mux * muy - mux - muy) / nd,
                 var_factor(nd) * cx.self * cy.self / (nd * nd * nd * nd), true, &rec);
    records[job.out] = rec;
  }
}

__global__ void __launch_bounds__(kStatThreads) hsic_perm_pair_kernel(int n, int max_rank,
                                                                       const double* __restrict__ factors,
                                                                       const HsicComponent* __restrict__ comps,
                                                                       const PairJob* __restrict__ pairs, int count,
                                                                       const int* __restrict__ perms, int replicates,
                                                                       RecordDev* __restrict__ records) {
  __shared__ double red[kStatThreads / 32];
  const int t = blockIdx.x;
  if (t >= count) return;
  const PairJob job = pairs[t];
  const HsicComponent cx = comps[job.left], cy = comps[job.right];
  const double* Gx = factors + static_cast<int64_t>(n) * max_rank * job.left;
  const double* Gy = factors + static_cast<int64_t>(n) * max_rank * job.right;
  const double nd = static_cast<double>(n);
  const double obs = hsic_cross(n, Gx, cx.rank, Gy, cy.rank, nullptr, red) / (nd * nd);
  int exceed = 1;
  for (int rep = 0; rep < replicates; ++rep) {
    const int* pi = perms + (static_cast<int64_t>(t) * replicates + rep) * n;
    const double s = hsic_cross(n, Gx, cx.rank, Gy, cy.rank, pi, red) / (nd * nd);
    if (s >= obs) ++exceed;
  }
  if (threadIdx.x == 0) {
    RecordDev rec;
    rec.statistic = obs;
    rec.mean = NAN;
    rec.variance = NAN;
    rec.p_value = static_cast<double>(exceed) / static_cast<double>(replicates + 1);
    rec.p_exact = rec.p_value;
    rec.status = kStatusOk;
    rec.flags = 0;
    records[job.out] = rec;
  }
}

__global__ void __launch_bounds__(kStatThreads) dcc_perm_pair_kernel(const double* __restrict__ residuals, int n,
                                                                      const int* __restrict__ comp_cols,
                                                                      const double* __restrict__ centre,
                                                                      const PairJob* __restrict__ pairs, int count,
                                                                      const int* __restrict__ perms, int replicates,
                                                                      RecordDev* __restrict__ records) {
  extern __shared__ double sm[];
  __shared__ double red[kStatThreads / 32];
  const int t = blockIdx.x;
  if (t >= count) return;
  const PairJob job = pairs[t];
  double* x = sm;
  double* cx = sm + n;
  double* y = sm + 2 * n;
  double* cy = sm + 3 * n;
  const double* xs = residuals + static_cast<int64_t>(n) * comp_cols[job.left];
  const double* ys = residuals + static_cast<int64_t>(n) * comp_cols[job.right];
  const double* cxs = centre + static_cast<int64_t>(n) * job.left;
  const double* cys = centre + static_cast<int64_t>(n) * job.right;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    x[i] = xs[i];
    cx[i] = cxs[i];
  }
  const double nd = static_cast<double>(n);
  double obs = 0.0;
  int exceed = 1;
  for (int rep = -1; rep < replicates; ++rep) {
    const int* pi = rep >= 0 ? perms + (static_cast<int64_t>(t) * replicates + rep) * n : nullptr;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int src = pi ? pi[i] : i;
      y[i] = ys[src];
      cy[i] = cys[src];
    }
    __syncthreads();
    double acc = 0.0;
    const int half = (n + 1) / 2;
    for (int tt = threadIdx.x; tt < half; tt += blockDim.x) {
      const int a = tt, b = n - 1 - tt;
      {
        const double xa = x[a], ya = y[a], ca = cx[a], da = cy[a];
        for (int j = a + 1; j < n; ++j) acc = fma(fabs(xa - x[j]) - ca - cx[j], fabs(ya - y[j]) - da - cy[j], acc);
      }
      if (b != a) {
        const double xb = x[b], yb = y[b], cb = cx[b], db = cy[b];
        for (int j = b + 1; j < n; ++j) acc = fma(fabs(xb - x[j]) - cb - cx[j], fabs(yb - y[j]) - db - cy[j], acc);
      }
    }
    double diag = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) diag += 4.0 * cx[i] * cy[i];
    const double s = (2.0 * block_sum256(acc, red) + block_sum256(diag, red)) / nd;
    if (rep < 0) obs = s;
    else if (s >= obs) ++exceed;
  }
  if (threadIdx.x == 0) {
    RecordDev rec;
    rec.statistic = obs;
    rec.mean = NAN;
    rec.variance = NAN;
    rec.p_value = static_cast<double>(exceed) / static_cast<double>(replicates + 1);
    rec.p_exact = rec.p_value;
    rec.status = kStatusOk;
    rec.flags = 0;
    records[job.out] = rec;
  }
}

// ------------------------------------------------------- FP64 peak probe

// 16 independent FMA chains per thread; the result is written so the chains
// are not removed.  Flops per launch: 2 * 16 * iters * threads.
__global__ void __launch_bounds__(256) fp64_fma_kernel(double* __restrict__ out, int iters, double a, double b) {
  double x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = 1e-3 * (threadIdx.x + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t launch_fp64_peak(double* out, int blocks, int iters, cudaStream_t stream) {
  fp64_fma_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.9999999, 1e-7);
  return cudaGetLastError();
}

// ------------------------------------------------------------- launchers

// legacy Lanczos: r (sorted), q, w (n doubles each) and the sort permutation (n ints)
size_t legacy_smem_bytes(int n) { return sizeof(double) * 3 * static_cast<size_t>(n) + sizeof(int) * static_cast<size_t>(n); }

// ------------------------------------------------------------ partition

__global__ void __launch_bounds__(1024) stat_partition_kernel(const int* __restrict__ defer_list,
                                                              const int* __restrict__ defer_count,
                                                              const FitJob* __restrict__ jobs, int ncomp,
                                                              const PairJob* __restrict__ pairs, int npairs,
                                                              int* __restrict__ late_col, int* __restrict__ part) {
  for (int c = threadIdx.x; c < ncomp; c += blockDim.x) late_col[c] = 0;
  if (threadIdx.x < 4) part[threadIdx.x] = 0;
  __syncthreads();
  const int deferred = defer_count ? *defer_count : 0;
  for (int d = threadIdx.x; d < deferred; d += blockDim.x) {
    const int col = jobs[defer_list[d]].out;
    if (col >= 0 && col < ncomp) late_col[col] = 1;
  }
  __syncthreads();
  int* early_comps = part + 4;
  int* late_comps = early_comps + ncomp;
  int* early_pairs = late_comps + ncomp;
  int* late_pairs = early_pairs + npairs;
  for (int c = threadIdx.x; c < ncomp; c += blockDim.x) {
    if (late_col[c]) late_comps[atomicAdd(part + 1, 1)] = c;
    else early_comps[atomicAdd(part + 0, 1)] = c;
  }
  for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
    const PairJob job = pairs[t];
    if (late_col[job.left] || late_col[job.right]) late_pairs[atomicAdd(part + 3, 1)] = t;
    else early_pairs[atomicAdd(part + 2, 1)] = t;
  }
}

cudaError_t launch_stat_partition(const int* defer_list, const int* defer_count, const FitJob* jobs, int ncomp,
                                  const PairJob* pairs, int npairs, int* late_col, int* part, cudaStream_t stream) {
  if (ncomp <= 0) return cudaSuccess;
  stat_partition_kernel<<<1, 1024, 0, stream>>>(defer_list, defer_count, jobs, ncomp, pairs, npairs, late_col, part);
  return cudaGetLastError();
}

__global__ void gamma_q_eval_kernel(const double* __restrict__ a, const double* __restrict__ x, int count,
                                    double* __restrict__ q, int* __restrict__ ok) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    int good = 0;
    q[i] = gamma_q(a[i], x[i], &good);
    ok[i] = good;
  }
}

cudaError_t launch_gamma_q_eval(const double* a, const double* x, int count, double* q, int* ok,
                                cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  gamma_q_eval_kernel<<<(count + 255) / 256, 256, 0, stream>>>(a, x, count, q, ok);
  return cudaGetLastError();
}

cudaError_t set_stat_limits(int n);

namespace {
// Largest n the statistic kernels' shared-memory limits were raised for, per
// device.  The limits only ever grow, so a call for a small n can never lower
// them under a launch for a larger n made by another thread.
std::mutex g_stat_limit_mu;
std::map<int, int> g_stat_limit_n;
}  // namespace

cudaError_t configure_stat_kernels(int n) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_stat_limit_mu);
  int& done = g_stat_limit_n[dev];
  if (n <= done) return cudaSuccess;
  if ((e = set_stat_limits(n)) == cudaSuccess) done = n;
  return e;
}

cudaError_t set_stat_limits(int n) {
  const int s2 = static_cast<int>(sizeof(double) * 2 * n);
  const int s3 = static_cast<int>(sizeof(double) * 3 * n);
  const int s4 = static_cast<int>(sizeof(double) * 4 * n);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(dcov_component_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s2)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(dcov_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s4)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(dcc_perm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s4)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(legacy_eigen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(legacy_smem_bytes(n)))) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(hsic_component_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, s3);
}

cudaError_t launch_dcov_components(const double* residuals, int n, const int* comp_cols, int count,
                                   double* centre, DcovComponent* comps, cudaStream_t stream, WorkList wl) {
  if (count <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * 2 * n;
  dcov_component_kernel<<<count, kStatThreads, smem, stream>>>(residuals, n, comp_cols, count, centre, comps, wl);
  return cudaGetLastError();
}

cudaError_t launch_dcov_pairs(const double* residuals, int n, const int* comp_cols, const double* centre,
                              const DcovComponent* comps, const PairJob* pairs, int count, RecordDev* records,
                              cudaStream_t stream, WorkList wl) {
  if (count <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * 4 * n;
  dcov_pair_kernel<<<count, kStatThreads, smem, stream>>>(residuals, n, comp_cols, centre, comps, pairs, count,
                                                           records, wl);
  return cudaGetLastError();
}

size_t legacy_eigen_workspace_doubles(int n, int ctas) {
  const size_t per = static_cast<size_t>(n) * (kLanczosMax + 1) + static_cast<size_t>(kLanczosMax) * 64 +
                     static_cast<size_t>(64) * 5 * kLanczosMax;
  return per * static_cast<size_t>(ctas);
}

cudaError_t launch_guard_select(const RecordDev* records, const PairJob* pairs, int count, int ncomp, int cap,
                                double lo, double hi, int* guard, cudaStream_t stream, WorkList wl, int append,
                                int* mark) {
  if (count <= 0) return cudaSuccess;
  if (append && !mark) return cudaErrorInvalidValue;
  guard_select_kernel<<<1, 1024, 0, stream>>>(records, pairs, count, ncomp, cap, lo, hi, guard, wl, append, mark);
  return cudaGetLastError();
}

cudaError_t launch_legacy_eigen(const double* residuals, int n, const int* comp_cols, const int* guard,
                                const int* slot_comps, int cap, int ctas, int num_col, double* workspace,
                                double* lowrank_vals, double* lowrank_vecs, int* status, cudaStream_t stream,
                                const int* slot_begin) {
  if (cap <= 0 || ctas <= 0) return cudaSuccess;
  if (num_col > 64) return cudaErrorInvalidValue;
  const size_t smem = legacy_smem_bytes(n);
  legacy_eigen_kernel<<<ctas, kStatThreads, smem, stream>>>(residuals, n, comp_cols, guard, slot_comps, cap,
                                                             num_col, workspace, lowrank_vals, lowrank_vecs, status,
                                                             slot_begin);
  return cudaGetLastError();
}

cudaError_t launch_legacy_pairs(int n, int num_col, const double* lowrank_vals, const double* lowrank_vecs,
                                const DcovComponent* comps, const int* guard, const int* guard_pairs,
                                const int* comp_slot, const PairJob* pairs, int count, RecordDev* records,
                                cudaStream_t stream, const int* list_begin) {
  if (count <= 0) return cudaSuccess;
  legacy_pair_kernel<<<count, kStatThreads, 0, stream>>>(n, num_col, lowrank_vals, lowrank_vecs, comps, guard,
                                                         guard_pairs, comp_slot, pairs, count, records, list_begin);
  return cudaGetLastError();
}

cudaError_t launch_hsic_components(const double* residuals, int n, const int* comp_cols, int count, int num_col,
                                   double sig, double* factors, HsicComponent* comps, cudaStream_t stream,
                                   WorkList wl) {
  if (count <= 0) return cudaSuccess;
  if (num_col > 64) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * 3 * n;
  hsic_component_kernel<<<count, kStatThreads, smem, stream>>>(residuals, n, comp_cols, count, num_col, 1.0 / sig,
                                                                factors, comps, wl);
  return cudaGetLastError();
}

cudaError_t launch_hsic_pairs(int n, int num_col, const double* factors, const HsicComponent* comps,
                              const PairJob* pairs, int count, RecordDev* records, cudaStream_t stream,
                              WorkList wl) {
  if (count <= 0) return cudaSuccess;
  hsic_pair_kernel<<<count, kStatThreads, 0, stream>>>(n, num_col, factors, comps, pairs, count, records, wl);
  return cudaGetLastError();
}

cudaError_t launch_hsic_perm_pairs(int n, int num_col, const double* factors, const HsicComponent* comps,
                                   const PairJob* pairs, int count, const int* perms, int replicates,
                                   RecordDev* records, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  hsic_perm_pair_kernel<<<count, kStatThreads, 0, stream>>>(n, num_col, factors, comps, pairs, count, perms,
                                                            replicates, records);
  return cudaGetLastError();
}

cudaError_t launch_dcc_perm_pairs(const double* residuals, int n, const int* comp_cols, const double* centre,
                                  const PairJob* pairs, int count, const int* perms, int replicates,
                                  RecordDev* records, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * 4 * n;
  dcc_perm_pair_kernel<<<count, kStatThreads, smem, stream>>>(residuals, n, comp_cols, centre, pairs, count, perms,
                                                               replicates, records);
  return cudaGetLastError();
}

}  // namespace fkpc
