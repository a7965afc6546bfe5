// WAN-PDAG orientation of a kernel-PC skeleton on the engine's regression and
// statistic kernels.
#pragma once

#include <functional>
#include <vector>

#include "runtime.h"

namespace fkpc {

struct OrientationTest {
  int reverse;           // 0: V's own regrVonPS; 1: the reverse test of a W in S
  int target;            // the regressed variable
  int other;             // the member of S tested against the residual
  std::vector<int> S;    // the subset
  std::vector<int> Z;    // S + parents(target), sorted: the residual's conditioning set
  double p_value;
  bool rejected;         // p_value < alpha
};

struct Orientation {
  std::vector<int> pdag;  // p*p column-major; pdag[i + p*j] = 1 and pdag[j + p*i] = 0 is i -> j
  int collider = 0, rule1 = 0, rule2 = 0, rule3 = 0, generalized = 0;
  int regrvonps_calls = 0;
  int residual_fits = 0, residual_cache_hits = 0;
  std::vector<OrientationTest> trace;
};

// One regrVonPS call's CI tests: p_values[k] for the test of (residual of
// target on Z, data[:, S[k]]).
using RegrVonPs = std::function<void(int target, const std::vector<int>& S, const std::vector<int>& Z,
                                     double* p_values)>;

// The orientation's graph logic over any CI evaluator.
Orientation orient_wanpdag(const RegrVonPs& eval, double alpha, int p, const int* adjacency,
                           const int* sepset_offsets, const int* sepset_values);

// Orients the skeleton (adjacency p*p column-major, sepsets CSR over cells
// i + p*j) of the data the engine has loaded; opt supplies alpha, the CI
// method (gamma methods), numCol, the HSIC sig and the selection.
Orientation orient_wanpdag(Engine& eng, const fkpc_options& opt, const double* data, int n, int p,
                           const int* adjacency, const int* sepset_offsets, const int* sepset_values);

}  // namespace fkpc
