// WAN-PDAG orientation of a kernel-PC skeleton (the step kpcalg's kpc()
// runs after the skeleton, kpcalg/R/kpc.R:137 -> kpcalg/R/udag2wanpdag.R:104-437,
// with kpc()'s defaults: no unfaithful-triple list, solve.confl = FALSE,
// rules 1-3).  The graph logic runs here on the host; every regrVonPS
// (kpcalg/R/regrvonps.R:17-39) runs on the GPU: the residual of V on
// S + parents(V) through the engine's regression, then the CI test of that
// residual against each member of S with no conditioning set through the
// engine's statistics.
//
// pdag(i, j) = 1 with pdag(j, i) = 0 is the edge i -> j; both 1 is an
// undirected edge.  Iteration orders are R's, since the orientation writes
// in place: which(M, arr.ind = TRUE) walks a matrix column by column and
// combn gives combinations in lexicographic order of positions.  The
// semantics are kpcalg's, which the reference's strict pipeline runs
// (fastkpc/R/fast_kpc.R:263-330 and :499-511): the subsets of V's
// neighbourhood listed before an accepted orientation are still tried after
// it, and rules 2 and 3 do not re-check that a - b is still undirected.
// Residuals are cached per (V, sorted conditioning set), as the reference's
// native engine does (fastkpc/src/regrvonps_native.cpp:60-100).
#include "orient.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace fkpc {
namespace {

class Orienter {
 public:
  Orienter(const RegrVonPs& eval, double alpha, int p, Orientation& out)
      : eval_(eval), alpha_(alpha), p_(p), g_(static_cast<size_t>(p) * p, 0), out_(out) {}

  int& at(std::vector<int>& m, int i, int j) { return m[static_cast<size_t>(i) * p_ + j]; }
  // i -> j; 1 when the matrix changed
  int orient(std::vector<int>& m, int i, int j) {
    const int changed = (at(m, i, j) != 1 || at(m, j, i) != 0) ? 1 : 0;
    at(m, i, j) = 1;
    at(m, j, i) = 0;
    return changed;
  }
  int get(const std::vector<int>& m, int i, int j) const { return m[static_cast<size_t>(i) * p_ + j]; }

  // (row, col) pairs with mask(row, col) in column-major order
  template <class F>
  std::vector<std::pair<int, int>> which(F mask) const {
    std::vector<std::pair<int, int>> out;
    for (int j = 0; j < p_; ++j)
      for (int i = 0; i < p_; ++i)
        if (mask(i, j)) out.emplace_back(i, j);
    return out;
  }

  // the k-subsets of v (R's combn; callers never ask for k > |v|, so R's
  // special case of a single value is the general path here)
  static std::vector<std::vector<int>> combn(const std::vector<int>& v, int k) {
    std::vector<std::vector<int>> out;
    if (k <= 0 || k > static_cast<int>(v.size())) return out;
    std::vector<int> idx(k);
    for (int i = 0; i < k; ++i) idx[i] = i;
    for (;;) {
      std::vector<int> c(k);
      for (int i = 0; i < k; ++i) c[i] = v[idx[i]];
      out.push_back(c);
      int i = k - 1;
      while (i >= 0 && idx[i] == static_cast<int>(v.size()) - k + i) --i;
      if (i < 0) break;
      ++idx[i];
      for (int j = i + 1; j < k; ++j) idx[j] = idx[j - 1] + 1;
    }
    return out;
  }

  std::vector<std::vector<int>> undirected(const std::vector<int>& pd) const {
    std::vector<std::vector<int>> nb(p_);
    for (int i = 0; i < p_; ++i)
      for (int j = 0; j < p_; ++j)
        if (get(pd, i, j) == 1 && get(pd, j, i) == 1) nb[i].push_back(j);
    return nb;
  }

  std::vector<int> parents(const std::vector<int>& pd, int v) const {
    std::vector<int> out;
    for (int i = 0; i < p_; ++i)
      if (get(pd, i, v) == 1 && get(pd, v, i) == 0) out.push_back(i);
    return out;
  }

  // kpcalg's checkImmor (udag2wanpdag.R:278-293)
  bool check_immor(const std::vector<int>& pd, int v, const std::vector<int>& S) const {
    auto und = [&](int a, int b) { return std::min(get(pd, a, b) + get(pd, b, a), 1); };
    if (S.size() > 1)
      for (size_t a = 0; a < S.size(); ++a)
        for (size_t b = 0; b < S.size(); ++b)
          if (a != b && und(S[a], S[b]) == 0 && und(S[b], S[a]) == 0) return false;
    const std::vector<int> par = parents(pd, v);
    int sum = 0;
    for (int a : par)
      for (int s : S) sum += und(a, s);
    return sum >= static_cast<int>(S.size() * par.size());
  }

  // rule 1 (udag2wanpdag.R:115-168): a -> b - c, a and c non-adjacent: b -> c
  int rule1(std::vector<int>& pd) {
    int count = 0;
    for (auto [a, b] : which([&](int i, int j) { return get(pd, i, j) == 1 && get(pd, j, i) == 0; })) {
      std::vector<int> isC;
      for (int c = 0; c < p_; ++c)
        if (get(pd, b, c) == 1 && get(pd, c, b) == 1 && get(pd, a, c) == 0 && get(pd, c, a) == 0) isC.push_back(c);
      for (int c : isC) count += orient(pd, b, c);
    }
    return count;
  }

  // rule 2 (:169-193): a - b with a chain a -> c -> b: a -> b
  int rule2(std::vector<int>& pd) {
    int count = 0;
    for (auto [a, b] : which([&](int i, int j) { return get(pd, i, j) == 1 && get(pd, j, i) == 1; })) {
      bool chain = false;
      for (int c = 0; c < p_; ++c)
        if (get(pd, a, c) == 1 && get(pd, c, a) == 0 && get(pd, c, b) == 1 && get(pd, b, c) == 0) chain = true;
      if (chain) count += orient(pd, a, b);
    }
    return count;
  }

  // rule 3 (:195-261): a - b, a - c1 -> b, a - c2 -> b, c1 and c2 non-adjacent: a -> b
  int rule3(std::vector<int>& pd) {
    int count = 0;
    for (auto [a, b] : which([&](int i, int j) { return get(pd, i, j) == 1 && get(pd, j, i) == 1; })) {
      std::vector<int> cs;
      for (int c = 0; c < p_; ++c)
        if (get(pd, a, c) == 1 && get(pd, c, a) == 1 && get(pd, c, b) == 1 && get(pd, b, c) == 0) cs.push_back(c);
      if (cs.size() < 2) continue;
      bool done = false;
      for (size_t i = 0; i < cs.size() && !done; ++i)
        for (size_t j = i + 1; j < cs.size() && !done; ++j)
          if (get(pd, cs[i], cs[j]) == 0 && get(pd, cs[j], cs[i]) == 0) {
            count += orient(pd, a, b);
            done = true;
          }
    }
    return count;
  }

  // kpcalg's regrVonPS (regrvonps.R:17-39): how many members s of S give
  // p < alpha for the test of (residual of V on S + parents(V), data[:, s])
  int regr_v_on_ps(const std::vector<int>& pd, int v, const std::vector<int>& S, int reverse) {
    ++out_.regrvonps_calls;
    std::vector<int> Z = S;
    for (int a : parents(pd, v)) Z.push_back(a);
    std::sort(Z.begin(), Z.end());
    std::vector<double> pv(S.size(), NAN);
    eval_(v, S, Z, pv.data());
    int count = 0;
    for (size_t k = 0; k < S.size(); ++k) {
      if (!(pv[k] == pv[k]))
        throw Error(FKPC_STATUS_NUMERIC, "orientation: CI test of variable " + std::to_string(v) + " failed");
      const bool rej = pv[k] < alpha_;
      out_.trace.push_back(OrientationTest{reverse, v, S[k], S, Z, pv[k], rej});
      if (rej) ++count;
    }
    return count;
  }

  std::vector<int> run(const int* adjacency, const int* sep_off, const int* sep_val) {
    for (int i = 0; i < p_; ++i)
      for (int j = 0; j < p_; ++j) at(g_, i, j) = (i != j && adjacency[i + static_cast<size_t>(p_) * j]) ? 1 : 0;
    std::vector<int> pd = g_;
    bool any = false;
    for (int v : g_) any = any || v;
    if (!any) return pd;
    auto in_sepset = [&](int a, int b, int y) {
      const size_t cell = static_cast<size_t>(a) + static_cast<size_t>(p_) * b;
      for (int k = sep_off[cell]; k < sep_off[cell + 1]; ++k)
        if (sep_val[k] == y) return true;
      return false;
    };
    // colliders x -> y <- z (udag2wanpdag.R:296-324)
    for (auto [x, y] : which([&](int i, int j) { return get(g_, i, j) == 1; }))
      for (int z = 0; z < p_; ++z) {
        if (z == x || get(g_, y, z) != 1) continue;
        if (get(g_, x, z) == 0 && !in_sepset(x, z, y) && !in_sepset(z, x, y)) {
          const int changed = orient(pd, x, y) | orient(pd, z, y);
          out_.collider += changed;
        }
      }
    // undirected neighbourhoods of growing size (:326-429)
    std::vector<std::vector<int>> nb = undirected(pd);
    std::vector<int> size(p_);
    for (int i = 0; i < p_; ++i) size[i] = static_cast<int>(nb[i].size());
    std::vector<char> updated(p_, 0);
    for (int s = 1; *std::max_element(size.begin(), size.end()) >= s; ++s) {
      for (int V = 0; V < p_; ++V) {
        int s2 = s;
        if (!(size[V] == s2 || (size[V] < s2 && updated[V]))) continue;
        s2 = size[V];
        while (s2 > 0) {
          const std::vector<std::vector<int>> subsets = combn(nb[V], s2);
          for (const auto& S : subsets) {
            if (!check_immor(pd, V, S)) continue;
            bool to_update = regr_v_on_ps(pd, V, S, 0) == 0;
            for (size_t k = 0; k < S.size() && to_update; ++k) {
              const int W = S[k];
              for (int s3 = size[W]; s3 > 0 && to_update; --s3)
                for (const auto& S2 : combn(nb[W], s3)) {
                  if (!to_update) break;  // the remaining tests cannot change the outcome
                  if (check_immor(pd, W, S2) && std::count(S2.begin(), S2.end(), V) == 1 &&
                      regr_v_on_ps(pd, W, S2, 1) == 0)
                    to_update = false;
                }
            }
            if (!to_update) continue;
            ++out_.generalized;
            for (int a : S) {
              at(pd, V, a) = 0;
              at(pd, a, V) = 1;
            }
            for (int u : nb[V])
              if (std::find(S.begin(), S.end(), u) == S.end()) {
                at(pd, u, V) = 0;
                at(pd, V, u) = 1;
              }
            s2 = 0;
            for (;;) {
              const std::vector<int> old = pd;
              out_.rule1 += rule1(pd);
              out_.rule2 += rule2(pd);
              out_.rule3 += rule3(pd);
              if (pd == old) break;
            }
            nb = undirected(pd);
            updated[V] = 1;
            for (int i = 0; i < p_; ++i) size[i] = static_cast<int>(nb[i].size());
          }
          --s2;
        }
      }
    }
    return pd;
  }

 private:
  const RegrVonPs& eval_;
  double alpha_;
  int p_;
  std::vector<int> g_;
  Orientation& out_;
};

}  // namespace

Orientation orient_wanpdag(const RegrVonPs& eval, double alpha, int p, const int* adjacency,
                           const int* sepset_offsets, const int* sepset_values) {
  Orientation out;
  Orienter o(eval, alpha, p, out);
  const std::vector<int> pd = o.run(adjacency, sepset_offsets, sepset_values);
  out.pdag.assign(static_cast<size_t>(p) * p, 0);
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j) out.pdag[i + static_cast<size_t>(p) * j] = pd[static_cast<size_t>(i) * p + j];
  return out;
}

Orientation orient_wanpdag(Engine& eng, const fkpc_options& opt, const double* data, int n, int p,
                           const int* adjacency, const int* sepset_offsets, const int* sepset_values) {
  // residuals per (target, sorted conditioning set), reused across calls
  std::map<std::pair<int, std::vector<int>>, std::vector<double>> residuals;
  int fits = 0, hits = 0;
  RegrVonPs eval = [&](int v, const std::vector<int>& S, const std::vector<int>& Z, double* p_values) {
    const size_t nn = static_cast<size_t>(n);
    std::vector<double> cols(nn * (1 + S.size()));
    auto key = std::make_pair(v, Z);
    auto hit = residuals.find(key);
    if (hit != residuals.end()) {
      ++hits;
      std::copy(hit->second.begin(), hit->second.end(), cols.begin());
    } else {
      int status = 0;
      eng.regress({v}, {Z}, cols.data(), nullptr, 0, &status, opt.selection);
      ++fits;
      if (status != 0)
        throw Error(FKPC_STATUS_NUMERIC, "orientation: residual fit of variable " + std::to_string(v) + " failed");
      residuals.emplace(key, std::vector<double>(cols.begin(), cols.begin() + nn));
    }
    for (size_t k = 0; k < S.size(); ++k)
      std::copy(data + nn * S[k], data + nn * (S[k] + 1), cols.begin() + nn * (k + 1));
    std::vector<int> left(S.size(), 0), right(S.size());
    for (size_t k = 0; k < S.size(); ++k) right[k] = static_cast<int>(k + 1);
    std::vector<fkpc_ci_record> rec(S.size());
    eng.statistics(cols.data(), static_cast<int>(1 + S.size()), left, right, nullptr, opt, rec.data());
    for (size_t k = 0; k < S.size(); ++k) p_values[k] = rec[k].p_value;
  };
  Orientation out = orient_wanpdag(eval, opt.alpha, p, adjacency, sepset_offsets, sepset_values);
  out.residual_fits = fits;
  out.residual_cache_hits = hits;
  return out;
}

}  // namespace fkpc
