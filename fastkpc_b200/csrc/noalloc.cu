// Exact-screen dCov gamma p-values without any device allocation.
//
// For callers that cannot call cudaMalloc: code running inside a host
// framework that owns every device allocation (a memory pool handed out by
// an R or JVM runtime, a plugin that may only use the buffers it is given),
// or code that must not allocate after start-up.  The caller passes device
// inputs and outputs; the scratch the two dCov kernels need between them --
// the row-centring constants and moments of each residual column and the
// pair jobs -- lives in one file-scope __device__ array of a fixed size
// (kScratchDoubles doubles, 8 MiB), which every GPU that loads the library
// keeps until the process exits.
//
// Host code must not use the array's name as a device address (on the host
// it names a host-side stand-in): every call looks the address up with
// cudaGetSymbolAddress on the current device and checks the result, so a
// context that was torn down and re-created (cudaDeviceReset) gets the new
// address.  The first call on a device loads the library's device code there;
// make it before any stream capture.  Every call shares the array, so calls
// that overlap on the GPU (different streams or threads at once) race on it;
// calls on one stream, one after another, are safe.  Each call writes every
// scratch value it reads before reading it, so nothing is left over from an
// earlier call.  The statistic kernels' shared-memory limits are only ever
// raised (never lowered), so these calls may run beside the library's other
// entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/fastkpc_b200.h"
#include "device.h"
#include "kernels.h"

namespace fkpc {
namespace {

constexpr size_t kScratchDoubles = static_cast<size_t>(1) << 20;  // 8 MiB
constexpr int kMaxN = 4096;  // the pair kernel stages 4n doubles in shared memory

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

static_assert(sizeof(fkpc_ci_record) == sizeof(RecordDev), "record layouts must match");

__global__ void noalloc_plan_kernel(const int* __restrict__ pairs, int count, int m, int* __restrict__ comp_cols,
                                    PairJob* __restrict__ jobs, int* __restrict__ bad) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) comp_cols[c] = c;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    const int a = pairs[2 * t], b = pairs[2 * t + 1];
    const bool ok = a >= 0 && a < m && b >= 0 && b < m;
    if (!ok) atomicExch(bad, 1);
    jobs[t] = PairJob{ok ? a : 0, ok ? b : 0, t, 0};
  }
}

// Device address of the scratch array on the current device.
cudaError_t scratch_address(double** out) {
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<double*>(ptr);
  return cudaSuccess;
}

}  // namespace
}  // namespace fkpc

extern "C" int fkpc_dcov_gamma_noalloc(const double* residuals, int n, int m, const int* pairs, int count,
                                       fkpc_ci_record* out, void* stream_handle) {
  using namespace fkpc;
  if (count < 0 || (count > 0 && (!residuals || !pairs || !out)))
    return fail(FKPC_STATUS_INVALID_ARGUMENT, "null pointer or negative pair count");
  if (n <= 5 || m < 1) return fail(FKPC_STATUS_INVALID_ARGUMENT, "residuals must be n x m with n > 5 and m >= 1");
  if (n > kMaxN) return fail(FKPC_STATUS_INVALID_ARGUMENT, "n exceeds 4096, the limit of the no-allocation path");
  // scratch: centring constants n*m, moments m (two doubles each), column map
  // m ints, pair jobs count (two doubles each), one flag
  const size_t need = static_cast<size_t>(n) * m + 2 * static_cast<size_t>(m) + (static_cast<size_t>(m) + 1) / 2 +
                      2 * static_cast<size_t>(count) + 1;
  if (need > kScratchDoubles)
    return fail(FKPC_STATUS_INVALID_ARGUMENT,
                "problem needs " + std::to_string(need) + " scratch doubles, more than the fixed " +
                    std::to_string(kScratchDoubles) + " (8 MiB) of the no-allocation path");
  if (count == 0) {  // nothing to evaluate: no device work
    set_last_error("");
    return FKPC_OK;
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
  double* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) return fail(FKPC_STATUS_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  double* centre = base;
  DcovComponent* comps = reinterpret_cast<DcovComponent*>(centre + static_cast<size_t>(n) * m);
  int* comp_cols = reinterpret_cast<int*>(comps + m);
  PairJob* jobs = reinterpret_cast<PairJob*>(base + static_cast<size_t>(n) * m + 2 * static_cast<size_t>(m) +
                                             (static_cast<size_t>(m) + 1) / 2);
  int* bad = reinterpret_cast<int*>(jobs + count);
  if ((e = cudaMemsetAsync(bad, 0, sizeof(int), stream)) != cudaSuccess)
    return fail(FKPC_STATUS_CUDA, std::string("clear flag: ") + cudaGetErrorString(e));
  noalloc_plan_kernel<<<(std::max(count, m) + 255) / 256, 256, 0, stream>>>(pairs, count, m, comp_cols, jobs, bad);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(FKPC_STATUS_CUDA, cudaGetErrorString(e));
  if ((e = configure_stat_kernels(n)) != cudaSuccess)
    return fail(FKPC_STATUS_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(e));
  if ((e = launch_dcov_components(residuals, n, comp_cols, m, centre, comps, stream)) != cudaSuccess)
    return fail(FKPC_STATUS_CUDA, cudaGetErrorString(e));
  if ((e = launch_dcov_pairs(residuals, n, comp_cols, centre, comps, jobs, count, reinterpret_cast<RecordDev*>(out),
                             stream)) != cudaSuccess)
    return fail(FKPC_STATUS_CUDA, cudaGetErrorString(e));
  int hbad = 0;
  if ((e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return fail(FKPC_STATUS_CUDA, cudaGetErrorString(e));
  if (hbad) return fail(FKPC_STATUS_INVALID_ARGUMENT, "pair index outside [0, m)");
  set_last_error("");
  return FKPC_OK;
}
