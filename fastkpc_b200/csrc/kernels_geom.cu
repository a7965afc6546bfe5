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
// in L2.  A zero column norm leaves R(k, k) = 0 (an identity reflector, Q
// still orthonormal); the fits' rank rule drops that direction, so status[d]
// stays 0.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "kernels.h"

namespace fkpc {

namespace {

constexpr int kGeomThreads = 256;
constexpr int kGeomWarps = kGeomThreads / 32;
constexpr int kGeomMaxQ = 560;  // additive designs up to |S| = 62
constexpr size_t kGeomSmemLimit = 220 * 1024;    // dynamic + static shared memory of one CTA
constexpr size_t kAdditiveStaticSmem = 14 * 1024;  // colsrc, vks, betas, red (13.2 KB) rounded up
constexpr size_t kSingleStaticSmem = 44 * 1024;   // R, Ri, T, A, V, ... (41.2 KB) rounded up

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

// X (n x q, column-major, at W) = Q R by Householder reflections, in place:
// on return W holds Q and R (ldr) the upper triangle (its lower triangle must
// be zero on entry).  Reflector k = I - beta v v', v = (x_k - alpha, x_{k+1},
// ...): rows > k of column k keep v until Q is formed, v_k and beta sit in
// vks / betas (q doubles each).  Returns true when a column norm was zero
// (rank deficient).  Called by the whole block.
static __device__ bool householder_inplace(double* __restrict__ W, int n, int q, double* R, int ldr, double* vks,
                                    double* betas, double* red) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
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
      // v = (vk, x_{k+1}, ...): the pivot row apart, two chains below it
      double d0 = lane == 0 ? vk * c[k] : 0.0, d1 = 0.0;
      int i = k + 1 + lane;
      for (; i + 32 < n; i += 64) {
        d0 += x[i] * c[i];
        d1 += x[i + 32] * c[i + 32];
      }
      if (i < n) d0 += x[i] * c[i];
      const double dot = warp_sum_g(d0 + d1) * beta;
      for (int r = k + 1 + lane; r < n; r += 32) c[r] -= dot * x[r];
      if (lane == 0) {
        c[k] -= dot * vk;
        R[k + static_cast<int64_t>(ldr) * j] = c[k];  // row k is final
      }
    }
    if (tid == 0) {
      R[k + static_cast<int64_t>(ldr) * k] = alpha;
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
      double d0 = 0.0, d1 = 0.0;
      int i = k + 1 + lane;
      for (; i + 32 < n; i += 64) {
        d0 += x[i] * c[i];
        d1 += x[i + 32] * c[i + 32];
      }
      if (i < n) d0 += x[i] * c[i];
      const double dot = warp_sum_g(d0 + d1) * beta;
      for (int r = k + 1 + lane; r < n; r += 32) c[r] -= dot * x[r];
      if (lane == 0) c[k] = -dot * vk;
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x)
      x[i] = i < k ? 0.0 : (i == k ? 1.0 - beta * vk * vk : -beta * vk * x[i]);
    __syncthreads();
  }
  return deficient;
}

// in_smem: the design's n x q working matrix lives in dynamic shared memory
// (n q doubles available) and Q is written to the arena at the end;
// otherwise it is factored in place in the arena (L2).
template <class J>
__global__ void __launch_bounds__(kGeomThreads) additive_geometry_kernel(int n, const J* __restrict__ jobs,
                                                                         int count, double* __restrict__ arena,
                                                                         int* __restrict__ status, int in_smem) {
  extern __shared__ double wsm[];
  __shared__ const double* colsrc[kGeomMaxQ];
  __shared__ double vks[kGeomMaxQ], betas[kGeomMaxQ];
  __shared__ double red[kGeomWarps];
  const int tid = threadIdx.x;
  for (int d = blockIdx.x; d < count; d += gridDim.x) {
    const J& job = jobs[d];
    const int q = job.q;
    double* Q = arena + job.basis;
    double* W = in_smem ? wsm : Q;
    double* R = arena + job.rmat;
    for (int c = tid; c < q; c += blockDim.x) {
      const double* src = nullptr;  // the intercept column
      for (int j = 0; j < job.m; ++j)
        if (c >= job.off[j] && c < job.off[j] + job.dim[j]) src = job.src[j] + static_cast<int64_t>(n) * (c - job.off[j]);
      colsrc[c] = src;
    }
    __syncthreads();
    const int64_t nq = static_cast<int64_t>(n) * q;
    for (int c = 0; c < q; ++c) {
      const double* s = colsrc[c];
      double* wc = W + static_cast<int64_t>(n) * c;
      for (int r = tid; r < n; r += blockDim.x) wc[r] = s ? s[r] : 1.0;
    }
    for (int idx = tid; idx < q * q; idx += blockDim.x) R[idx] = 0.0;
    __syncthreads();
    const bool deficient = householder_inplace(W, n, q, R, q, vks, betas, red);
    if (in_smem)
      for (int64_t idx = tid; idx < nq; idx += blockDim.x) Q[idx] = W[idx];
    if (job.rpack >= 0) {
      double* rp = arena + job.rpack;
      for (int idx = tid; idx < kWarpTri; idx += blockDim.x) rp[idx] = 0.0;
      __syncthreads();
      for (int idx = tid; idx < q * q; idx += blockDim.x) {
        const int t = idx % q, c = idx / q;
        if (t <= c) rp[packed_row(t, c)] = R[idx];
      }
    }
    // a zero column (R(k, k) = 0, an identity reflector) is left to the fits,
    // whose rank rule drops the direction it leaves in the augmented system
    (void)deficient;
    if (tid == 0) status[d] = 0;
    __syncthreads();
  }
}

// Single-penalty designs (|S| <= 2): X = [1 | B] with one penalty S on the
// smooth's columns (fastkpc/src/full_cuda_ci_one_call.cpp:1869-1947 builds
// this geometry from the Gram Cholesky; here from the QR).  X = Q R, the
// whitened penalty R^-T S R^-1 = V diag(e) V' (parallel Jacobi, at most 100
// sweeps), and the fit kernels' inputs QW = Q V and the spectrum e
// (descending; zero beyond the penalty rank).  status[d]: 1 rank deficient,
// 2 Jacobi did not converge.
__global__ void __launch_bounds__(kGeomThreads) single_geometry_kernel(int n, const SingleGeomJob* __restrict__ jobs,
                                                                       int count, double* __restrict__ arena,
                                                                       int* __restrict__ status, int in_smem) {
  extern __shared__ double wsm[];
  constexpr int Q = kMaxSingleQ;
  constexpr int LA = Q + 1;  // padded leading dimension of the Jacobi matrices
  __shared__ double Rs[Q * Q], Ri[Q * Q], T[Q * Q];
  __shared__ double A[Q * LA], Vs[Q * LA];
  __shared__ double vks[Q], betas[Q], red[kGeomWarps];
  __shared__ int order[Q];
  __shared__ int jacobi_ok;
  __shared__ int rot_p[Q / 2 + 1], rot_q[Q / 2 + 1];
  __shared__ double rot_c[Q / 2 + 1], rot_s[Q / 2 + 1];
  const int tid = threadIdx.x;
  for (int d = blockIdx.x; d < count; d += gridDim.x) {
    const SingleGeomJob& job = jobs[d];
    const int q = job.q, dim = q - 1;
    double* QW = arena + job.basis;
    double* W = in_smem ? wsm : QW;
    const double* B = job.src;
    const double* S = job.pen;
    for (int r = tid; r < n; r += blockDim.x) W[r] = 1.0;
    for (int c = 1; c < q; ++c) {
      const double* bc = B + static_cast<int64_t>(n) * (c - 1);
      double* wc = W + static_cast<int64_t>(n) * c;
      for (int r = tid; r < n; r += blockDim.x) wc[r] = bc[r];
    }
    for (int idx = tid; idx < q * q; idx += blockDim.x) {
      Rs[idx] = 0.0;
      Ri[idx] = 0.0;
    }
    __syncthreads();
    const bool deficient = householder_inplace(W, n, q, Rs, q, vks, betas, red);
    if (deficient) {
      if (tid == 0) status[d] = 1;
      __syncthreads();
      continue;  // uniform: every thread holds the same flag
    }
    // Ri = R^-1, one column per thread, back substitution
    if (tid < q) {
      const int c = tid;
      Ri[c + q * c] = 1.0 / Rs[c + q * c];
      for (int r = c - 1; r >= 0; --r) {
        double acc = 0.0;
        for (int t = r + 1; t <= c; ++t) acc += Rs[r + q * t] * Ri[t + q * c];
        Ri[r + q * c] = -acc / Rs[r + q * r];
      }
    }
    __syncthreads();
    // T = S_full Ri (S_full: S on rows / columns 1..q-1), then A = Ri' T
    for (int idx = tid; idx < q * q; idx += blockDim.x) {
      const int r = idx % q, c = idx / q;
      double acc = 0.0;
      if (r > 0)
        for (int t = 1; t < q; ++t) acc += S[(r - 1) + static_cast<int64_t>(dim) * (t - 1)] * Ri[t + q * c];
      T[idx] = acc;
    }
    __syncthreads();
    for (int idx = tid; idx < q * q; idx += blockDim.x) {
      const int r = idx % q, c = idx / q;
      double acc = 0.0;
      for (int t = 0; t < q; ++t) acc += Ri[t + q * r] * T[t + q * c];
      A[r + LA * c] = acc;
    }
    __syncthreads();
    for (int idx = tid; idx < q * q; idx += blockDim.x) {
      const int r = idx % q, c = idx / q;
      if (r > c) {
        const double v = 0.5 * (A[r + LA * c] + A[c + LA * r]);
        A[r + LA * c] = v;
        A[c + LA * r] = v;
      }
    }
    __syncthreads();
    // Jacobi with the round-robin (circle) ordering: in each round the
    // index pairs are disjoint, so their rotations commute and are applied
    // together -- angles from the round's A, then all column updates (A J,
    // V J), then all row updates (J' A).  A sweep is Qe - 1 rounds over
    // Qe = q rounded up to even (the odd index out sits out the round).
    for (int idx = tid; idx < q * q; idx += blockDim.x) Vs[idx % q + LA * (idx / q)] = idx % q == idx / q ? 1.0 : 0.0;
    __syncthreads();
    const int qe = q + (q & 1);
    const int npair = qe / 2;
    bool conv = false;
    for (int sweep = 0; sweep < 100 && !conv; ++sweep) {
      double off = 0.0, diag = 0.0;
      for (int idx = tid; idx < q * q; idx += blockDim.x) {
        const int r = idx % q, c = idx / q;
        const double v = A[r + LA * c];
        if (r == c) diag += v * v;
        else off += v * v;
      }
      off = block_sum_g(off, red);
      __syncthreads();
      diag = block_sum_g(diag, red);
      if (off <= 1e-32 * diag || off == 0.0) {
        conv = true;
        break;
      }
      for (int round = 0; round < qe - 1; ++round) {
        if (tid < npair) {
          int a, b;
          if (tid == 0) {
            a = round;
            b = qe - 1;
          } else {
            a = (round + tid) % (qe - 1);
            b = (round - tid + qe - 1) % (qe - 1);
          }
          const int pp = a < b ? a : b, qq = a < b ? b : a;
          double cs = 1.0, sn = 0.0;
          if (qq < q) {
            const double apq = A[pp + LA * qq];
            if (apq != 0.0) {
              const double app = A[pp + LA * pp], aqq = A[qq + LA * qq];
              const double theta = (aqq - app) / (2.0 * apq);
              const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
              cs = 1.0 / sqrt(t * t + 1.0);
              sn = t * cs;
            }
          }
          rot_p[tid] = pp;
          rot_q[tid] = qq;
          rot_c[tid] = cs;
          rot_s[tid] = sn;
        }
        __syncthreads();
        // columns: A J and V J (pair i, row k)
        for (int idx = tid; idx < npair * q; idx += blockDim.x) {
          const int i = idx / q, k = idx % q;
          const int pp = rot_p[i], qq = rot_q[i];
          if (qq >= q || rot_s[i] == 0.0) continue;
          const double cs = rot_c[i], sn = rot_s[i];
          const double akp = A[k + LA * pp], akq = A[k + LA * qq];
          A[k + LA * pp] = cs * akp - sn * akq;
          A[k + LA * qq] = sn * akp + cs * akq;
          const double vkp = Vs[k + LA * pp], vkq = Vs[k + LA * qq];
          Vs[k + LA * pp] = cs * vkp - sn * vkq;
          Vs[k + LA * qq] = sn * vkp + cs * vkq;
        }
        __syncthreads();
        // rows: J' A (pair i, column k)
        for (int idx = tid; idx < npair * q; idx += blockDim.x) {
          const int i = idx / q, k = idx % q;
          const int pp = rot_p[i], qq = rot_q[i];
          if (qq >= q || rot_s[i] == 0.0) continue;
          const double cs = rot_c[i], sn = rot_s[i];
          const double apk = A[pp + LA * k], aqk = A[qq + LA * k];
          A[pp + LA * k] = cs * apk - sn * aqk;
          A[qq + LA * k] = sn * apk + cs * aqk;
        }
        __syncthreads();
        if (tid < npair && rot_q[tid] < q) {  // as the serial sweep: a_pq is zero after its rotation
          A[rot_p[tid] + LA * rot_q[tid]] = 0.0;
          A[rot_q[tid] + LA * rot_p[tid]] = 0.0;
        }
        __syncthreads();
      }
    }
    // descending eigenvalues; equal values: the higher index first
    if (tid < q) {
      const double li = A[tid + LA * tid];
      int pos = 0;
      for (int j = 0; j < q; ++j) {
        const double lj = A[j + LA * j];
        pos += (lj > li || (lj == li && j > tid)) ? 1 : 0;
      }
      order[pos] = tid;
    }
    if (tid == 0) jacobi_ok = conv ? 1 : 0;
    __syncthreads();
    if (!jacobi_ok) {
      if (tid == 0) status[d] = 2;
      __syncthreads();
      continue;
    }
    double* spec = arena + job.spec;
    if (tid < q) {
      const double lv = A[order[tid] + LA * order[tid]];
      spec[tid] = tid < job.rank ? fmax(0.0, lv) : 0.0;
    }
    // T = V sorted by descending eigenvalue
    for (int idx = tid; idx < q * q; idx += blockDim.x) {
      const int r = idx % q, c = idx / q;
      T[idx] = Vs[r + LA * order[c]];
    }
    __syncthreads();
    // QW = Q V, a row per thread (in place when W is the arena slot)
    for (int r = tid; r < n; r += blockDim.x) {
      double qrow[Q];
#pragma unroll
      for (int t = 0; t < Q; ++t) qrow[t] = t < q ? W[r + static_cast<int64_t>(n) * t] : 0.0;
#pragma unroll 4
      for (int c = 0; c < q; ++c) {
        double acc = 0.0;
#pragma unroll
        for (int t = 0; t < Q; ++t)
          if (t < q) acc += qrow[t] * T[t + q * c];
        QW[r + static_cast<int64_t>(n) * c] = acc;
      }
    }
    if (tid == 0) status[d] = 0;
    __syncthreads();
  }
}

namespace {

// Dynamic shared memory for an n x max_q working matrix, or 0 when it does
// not fit beside the static arrays (the arena is the working set then).
size_t geometry_smem(int n, int max_q, size_t static_bytes) {
  const size_t bytes = sizeof(double) * static_cast<size_t>(n) * max_q;
  return bytes + static_bytes <= kGeomSmemLimit ? bytes : 0;
}

template <class K>
cudaError_t geometry_launch_shape(K kernel, size_t smem, int count, int* ctas) {
  if (smem > 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }
  int per_sm = 4;  // CTAs resident per SM
  if (smem > 0) {
    per_sm = static_cast<int>(kGeomSmemLimit / (smem + 2048));
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
  }
  const int cap = 148 * per_sm;
  *ctas = count < cap ? count : cap;
  return cudaSuccess;
}

}  // namespace

cudaError_t launch_single_geometry(int n, const SingleGeomJob* jobs, int count, double* arena, int* status,
                                   cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  if (n <= kMaxSingleQ) return cudaErrorInvalidValue;
  const size_t smem = geometry_smem(n, kMaxSingleQ, kSingleStaticSmem);
  int ctas = 0;
  cudaError_t e = geometry_launch_shape(single_geometry_kernel, smem, count, &ctas);
  if (e != cudaSuccess) return e;
  single_geometry_kernel<<<ctas, kGeomThreads, smem, stream>>>(n, jobs, count, arena, status, smem > 0 ? 1 : 0);
  return cudaGetLastError();
}

template <class J>
cudaError_t launch_additive_geometry_t(int n, const J* jobs, int count, int max_q, double* arena, int* status,
                                       cudaStream_t stream) {
  if (count <= 0) return cudaSuccess;
  if (n < 2 || max_q < 1 || max_q > kGeomMaxQ || max_q >= n) return cudaErrorInvalidValue;
  const size_t smem = geometry_smem(n, max_q, kAdditiveStaticSmem);
  int ctas = 0;
  cudaError_t e = geometry_launch_shape(additive_geometry_kernel<J>, smem, count, &ctas);
  if (e != cudaSuccess) return e;
  additive_geometry_kernel<J><<<ctas, kGeomThreads, smem, stream>>>(n, jobs, count, arena, status, smem > 0 ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_additive_geometry(int n, const GeomJob* jobs, int count, int max_q, double* arena, int* status,
                                     cudaStream_t stream) {
  return launch_additive_geometry_t(n, jobs, count, max_q, arena, status, stream);
}

cudaError_t launch_additive_geometry(int n, const WideGeomJob* jobs, int count, int max_q, double* arena,
                                     int* status, cudaStream_t stream) {
  return launch_additive_geometry_t(n, jobs, count, max_q, arena, status, stream);
}

}  // namespace fkpc
