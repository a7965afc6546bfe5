// Geometry of the additive (|S| >= 3) designs on the device.
//
// An additive design is X = [1 | B_{s_1} | ... | B_{s_m}], the univariate
// thin-plate bases of its conditioning variables side by side
// (fastkpc/src/full_cuda_ci_native_setup.cpp:1188-1320, 1384-1417), and the
// fit kernels need its thin QR factors, Q explicit and R upper triangular.
// The reference's geometry step (full_cuda_ci_native_setup.cpp:1418-1558)
// factors X with LAPACK's pivoted dgeqp3 (:881-940); the GCV quantities
// depend only on the column space and on R'R = X'X, so the unpivoted
// Householder factorisation here serves the fits equally.  The host
// keeps only the small per-variable pieces (bases, penalty roots, column
// norms for initial.sp); additive_geometry_kernel gathers X from a table of
// the bases straight into the design's Q slot of the arena, factors it there
// by Householder reflections, writes R (and the row-packed R of the warp fit
// class), and forms Q in place by backward accumulation.
//
// One CTA per design (grid-stride).  Reflector k: a block reduction for the
// column norm, then warp per trailing column (dot product and update over the
// rows, coalesced).  The working set (n x q doubles, ~150 KB at n = 500) stays
// in L2.  A zero column norm marks the design rank deficient in status[d].
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "kernels.h"

namespace fkpc {

namespace {

constexpr int kGeomThreads = 256;
constexpr int kGeomWarps = kGeomThreads / 32;
constexpr int kGeomMaxQ = 112;

__device__ __forceinline__ double warp_sum_g(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; every thread gets the same value (fixed order).
__device__ double block_sum_g(double v, double* red) {
  v = warp_sum_g(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < kGeomWarps; ++w) s += red[w];
  return s;
}

}  // namespace

__global__ void __launch_bounds__(kGeomThreads) additive_geometry_kernel(const double* __restrict__ table, int n,
                                                                         const GeomJob* __restrict__ jobs, int count,
                                                                         double* __restrict__ arena,
                                                                         int* __restrict__ status) {
  __shared__ int64_t colsrc[kGeomMaxQ];
  __shared__ double vks[kGeomMaxQ], betas[kGeomMaxQ];
  __shared__ double red[kGeomWarps];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int d = blockIdx.x; d < count; d += gridDim.x) {
    const GeomJob& job = jobs[d];
    const int q = job.q;
    double* W = arena + job.basis;
    double* R = arena + job.rmat;
    if (tid < q) {
      int64_t src = -1;  // the intercept column
      for (int j = 0; j < job.m; ++j)
        if (tid >= job.off[j] && tid < job.off[j] + job.dim[j])
          src = job.src[j] + static_cast<int64_t>(n) * (tid - job.off[j]);
      colsrc[tid] = src;
    }
    __syncthreads();
    const int64_t nq = static_cast<int64_t>(n) * q;
    for (int64_t idx = tid; idx < nq; idx += blockDim.x) {
      const int r = static_cast<int>(idx % n), c = static_cast<int>(idx / n);
      const int64_t s = colsrc[c];
      W[idx] = s < 0 ? 1.0 : table[s + r];
    }
    for (int idx = tid; idx < q * q; idx += blockDim.x) R[idx] = 0.0;
    __syncthreads();
    // factorisation: reflector k = I - beta v v', v = (x_k - alpha, x_{k+1}, ...);
    // rows > k of column k keep v, v_k and beta go to shared memory
    bool deficient = false;
    for (int k = 0; k < q; ++k) {
      const double* x = W + static_cast<int64_t>(n) * k;
      double part = 0.0;
      for (int i = k + tid; i < n; i += blockDim.x) part += x[i] * x[i];
      const double norm2 = block_sum_g(part, red);
      const double norm = sqrt(norm2);
      const double xk = x[k];
      double alpha = 0.0, vk = 0.0, beta = 0.0;
      if (norm == 0.0) {
        deficient = true;
      } else {
        alpha = xk >= 0.0 ? -norm : norm;
        vk = xk - alpha;
        beta = 2.0 / (norm2 - xk * xk + vk * vk);
      }
      for (int j = k + 1 + warp; j < q; j += kGeomWarps) {
        double* c = W + static_cast<int64_t>(n) * j;
        double dot = 0.0;
        for (int i = k + lane; i < n; i += 32) dot += (i == k ? vk : x[i]) * c[i];
        dot = warp_sum_g(dot) * beta;
        for (int i = k + lane; i < n; i += 32) c[i] -= dot * (i == k ? vk : x[i]);
        if (lane == 0) R[k + static_cast<int64_t>(q) * j] = c[k];  // row k is final
      }
      if (tid == 0) {
        R[k + static_cast<int64_t>(q) * k] = alpha;
        vks[k] = vk;
        betas[k] = beta;
      }
      __syncthreads();
    }
    // Q = H_0 ... H_{q-1} [I; 0], accumulated backwards in place.  Before step
    // k, column j > k is zero in rows <= k, so its update starts at row k + 1
    // and row k receives -dot v_k.
    for (int k = q - 1; k >= 0; --k) {
      double* x = W + static_cast<int64_t>(n) * k;
      const double vk = vks[k], beta = betas[k];
      for (int j = k + 1 + warp; j < q; j += kGeomWarps) {
        double* c = W + static_cast<int64_t>(n) * j;
        double dot = 0.0;
        for (int i = k + 1 + lane; i < n; i += 32) dot += x[i] * c[i];
        dot = warp_sum_g(dot) * beta;
        for (int i = k + 1 + lane; i < n; i += 32) c[i] -= dot * x[i];
        if (lane == 0) c[k] = -dot * vk;
      }
      __syncthreads();
      for (int i = tid; i < n; i += blockDim.x)
        x[i] = i < k ? 0.0 : (i == k ? 1.0 - beta * vk * vk : -beta * vk * x[i]);
      __syncthreads();
    }
    if (job.rpack >= 0) {
      double* rp = arena + job.rpack;
      for (int idx = tid; idx < kWarpTri; idx += blockDim.x) rp[idx] = 0.0;
      __syncthreads();
      for (int idx = tid; idx < q * q; idx += blockDim.x) {
        const int t = idx % q, c = idx / q;
        if (t <= c) rp[packed_row(t, c)] = R[idx];
      }
    }
    if (tid == 0) status[d] = deficient ? 1 : 0;
    __syncthreads();
  }
}

cudaError_t launch_additive_geometry(const double* table, int n, const GeomJob* jobs, int count, int max_q,
                                     double* arena, int* status, cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  if (n < 2 || max_q < 1 || max_q > kGeomMaxQ || max_q >= n) return cudaErrorInvalidValue;
  const int ctas = count < 4 * 148 ? count : 4 * 148;
  additive_geometry_kernel<<<ctas, kGeomThreads, 0, stream>>>(table, n, jobs, count, arena, status);
  return cudaGetLastError();
}

}  // namespace fkpc
