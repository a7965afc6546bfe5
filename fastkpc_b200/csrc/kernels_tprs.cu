// Thin-plate set-up on the device: the Lanczos part of the top-k eigen problem
// of the eta matrix of every bivariate (|S| = 2) design of a level.
//
// mgcv's tp basis for d = 2 (m = 2, k = 30) needs the k largest-magnitude
// eigenpairs of E_ij = eta(|u_i - u_j|), eta(r) = r^2 log(r) / (8 pi), over the
// unique locations u (fastkpc/src/full_cuda_ci_native_setup.cpp:114-152, 303).
// On the host that is about 10 ms of Lanczos per design, hundreds of designs
// per level.  tprs_lanczos_kernel: one CTA per design (grid-stride over the
// level's designs); it builds E in its own global workspace, then runs a
// fixed number of Lanczos steps with full re-orthogonalisation (classical
// Gram-Schmidt, two passes, as the host) from the host's deterministic start
// vector.  The basis V and the tridiagonal (alpha, beta) go back to the host,
// which takes the Ritz pairs, checks their residuals and finishes the basis
// (ritz_from_lanczos, tprs_finish); a design whose Ritz pairs have not
// converged is rebuilt on the host.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "kernels.h"

namespace fkpc {

namespace {

constexpr int kTprsThreads = 256;

__device__ __forceinline__ double warp_sum_t(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum_t(double v, double* red) {
  v = warp_sum_t(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

}  // namespace

// u: the designs' unique locations, design d at u + uoff[d] (nus[d] x 2,
// column-major).  V: design d's basis at V + voff[d] (nus[d] x steps).
// alpha / beta: count x steps.  done[d]: steps taken (fewer when the Krylov
// space became invariant).  ews: per-CTA workspace of ews_stride doubles
// (>= max nus^2).  Dynamic shared memory: 2 x max nus doubles.
__global__ void __launch_bounds__(kTprsThreads) tprs_lanczos_kernel(
    const double* __restrict__ u, const int64_t* __restrict__ uoff, const int* __restrict__ nus, int count,
    int steps, double eta0, double* __restrict__ ews, int64_t ews_stride, double* __restrict__ V,
    const int64_t* __restrict__ voff, double* __restrict__ alpha, double* __restrict__ beta, int* __restrict__ done) {
  extern __shared__ double sm[];
  __shared__ double red[kTprsThreads / 32];
  __shared__ double coef[kTprsMaxSteps];
  __shared__ double scal[2];
  const int tid = threadIdx.x;
  for (int d = blockIdx.x; d < count; d += gridDim.x) {
    const int nu = nus[d];
    const double* ux = u + uoff[d];
    const double* uy = ux + nu;
    double* E = ews + ews_stride * blockIdx.x;
    double* Vd = V + voff[d];
    double* q = sm;
    double* w = sm + nu;
    // E_ij = eta0 log(r2) / 2 * r2 (the host's order of operations)
    const int64_t nn = static_cast<int64_t>(nu) * nu;
    for (int64_t idx = tid; idx < nn; idx += blockDim.x) {
      const int i = static_cast<int>(idx % nu), j = static_cast<int>(idx / nu);
      const double dx = ux[i] - ux[j], dy = uy[i] - uy[j];
      const double r2 = dx * dx + dy * dy;
      double v = 0.0;
      if (r2 > 0.0) {
        v = eta0;
        v *= log(r2) * 0.5;
        v *= r2;
      }
      E[idx] = v;
    }
    if (tid == 0) {
      unsigned long state = 1;
      double nrm = 0.0;
      for (int i = 0; i < nu; ++i) {
        state = (state * 106UL + 1283UL) % 6075UL;
        const double v = static_cast<double>(state) / 6075.0 - 0.5;
        q[i] = v;
        nrm += v * v;
      }
      scal[0] = sqrt(nrm);
    }
    __syncthreads();
    for (int i = tid; i < nu; i += blockDim.x) Vd[i] = q[i] / scal[0];
    __syncthreads();
    double anorm = 0.0, bprev = 0.0;
    int taken = 0;
    for (int j = 0; j < steps; ++j) {
      const double* vj = Vd + static_cast<int64_t>(nu) * j;
      for (int i = tid; i < nu; i += blockDim.x) q[i] = vj[i];
      __syncthreads();
      // w = E q: thread per row, four chains, coalesced column walk of E
      double part = 0.0;
      for (int i = tid; i < nu; i += blockDim.x) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int t = 0;
        for (; t + 3 < nu; t += 4) {
          s0 += E[i + static_cast<int64_t>(nu) * t] * q[t];
          s1 += E[i + static_cast<int64_t>(nu) * (t + 1)] * q[t + 1];
          s2 += E[i + static_cast<int64_t>(nu) * (t + 2)] * q[t + 2];
          s3 += E[i + static_cast<int64_t>(nu) * (t + 3)] * q[t + 3];
        }
        for (; t < nu; ++t) s0 += E[i + static_cast<int64_t>(nu) * t] * q[t];
        const double s = (s0 + s1) + (s2 + s3);
        w[i] = s;
        part += q[i] * s;
      }
      const double a = block_sum_t(part, red);
      const double* vp = j > 0 ? Vd + static_cast<int64_t>(nu) * (j - 1) : nullptr;
      for (int i = tid; i < nu; i += blockDim.x) {
        double v = w[i] - a * q[i];
        if (vp) v -= bprev * vp[i];
        w[i] = v;
      }
      __syncthreads();
      // full re-orthogonalisation, two passes
      for (int pass = 0; pass < 2; ++pass) {
        const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
        for (int b0 = 4 * warp; b0 <= j; b0 += 4 * nwarps) {
          const double* v0 = Vd + static_cast<int64_t>(nu) * b0;
          const bool h1 = b0 + 1 <= j, h2 = b0 + 2 <= j, h3 = b0 + 3 <= j;
          double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll 4
          for (int i = lane; i < nu; i += 32) {
            const double wi = w[i];
            const double x0 = v0[i];
            const double x1 = h1 ? v0[i + nu] : 0.0;
            const double x2 = h2 ? v0[i + 2 * static_cast<int64_t>(nu)] : 0.0;
            const double x3 = h3 ? v0[i + 3 * static_cast<int64_t>(nu)] : 0.0;
            s0 += wi * x0;
            s1 += wi * x1;
            s2 += wi * x2;
            s3 += wi * x3;
          }
          s0 = warp_sum_t(s0);
          s1 = warp_sum_t(s1);
          s2 = warp_sum_t(s2);
          s3 = warp_sum_t(s3);
          if (lane == 0) {
            coef[b0] = s0;
            if (h1) coef[b0 + 1] = s1;
            if (h2) coef[b0 + 2] = s2;
            if (h3) coef[b0 + 3] = s3;
          }
        }
        __syncthreads();
        for (int i = tid; i < nu; i += blockDim.x) {
          double s0 = w[i], s1 = 0.0, s2 = 0.0, s3 = 0.0;
          int b = 0;
          for (; b + 7 <= j; b += 8) {
            double x[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) x[t] = Vd[i + static_cast<int64_t>(nu) * (b + t)];
            s0 -= coef[b] * x[0] + coef[b + 4] * x[4];
            s1 -= coef[b + 1] * x[1] + coef[b + 5] * x[5];
            s2 -= coef[b + 2] * x[2] + coef[b + 6] * x[6];
            s3 -= coef[b + 3] * x[3] + coef[b + 7] * x[7];
          }
          for (; b <= j; ++b) s0 -= coef[b] * Vd[i + static_cast<int64_t>(nu) * b];
          w[i] = (s0 + s1) + (s2 + s3);
        }
        __syncthreads();
      }
      double nn2 = 0.0;
      for (int i = tid; i < nu; i += blockDim.x) nn2 += w[i] * w[i];
      const double bj = sqrt(block_sum_t(nn2, red));
      anorm = fmax(anorm, fabs(a) + bj + bprev);
      if (tid == 0) {
        alpha[static_cast<int64_t>(d) * steps + j] = a;
        beta[static_cast<int64_t>(d) * steps + j] = bj;
      }
      taken = j + 1;
      if (bj <= 1e-15 * anorm) break;  // invariant Krylov space: the Ritz pairs are exact
      if (j + 1 < steps) {
        double* vn = Vd + static_cast<int64_t>(nu) * (j + 1);
        for (int i = tid; i < nu; i += blockDim.x) vn[i] = w[i] / bj;
      }
      bprev = bj;
      __syncthreads();
    }
    if (tid == 0) done[d] = taken;
    __syncthreads();
  }
}

cudaError_t launch_tprs_lanczos(const double* u, const int64_t* uoff, const int* nus, int count, int nu_max,
                                int steps, double eta0, double* ews, int64_t ews_stride, int ctas, double* V,
                                const int64_t* voff, double* alpha, double* beta, int* done, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  if (steps < 1 || steps > kTprsMaxSteps || ctas < 1) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * 2 * static_cast<size_t>(nu_max);
  cudaError_t e = cudaFuncSetAttribute(tprs_lanczos_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  tprs_lanczos_kernel<<<ctas, kTprsThreads, smem, stream>>>(u, uoff, nus, count, steps, eta0, ews, ews_stride, V,
                                                             voff, alpha, beta, done);
  return cudaGetLastError();
}

}  // namespace fkpc
