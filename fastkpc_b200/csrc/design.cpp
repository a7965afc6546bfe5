// Thin-plate / additive design setup.  Follows mgcv 1.9-1's s() construction
// as the reference's native setup restates it
// (fastkpc/src/full_cuda_ci_native_setup.cpp:690-858 smooth, :621-688
// centering constraint, :1188-1317 assembly, :1019-1127 initial.sp), with
// the eigenpairs from this library's own Lanczos solver.
#include "design.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

#include "hostla.h"

namespace fkpc {

double r_mean(const double* v, int n) {
  long double m = 0.0L;
  for (int i = 0; i < n; ++i) m += v[i];
  m /= static_cast<long double>(n);
  long double c = 0.0L;
  for (int i = 0; i < n; ++i) c += static_cast<long double>(v[i]) - m;
  m += c / static_cast<long double>(n);
  return static_cast<double>(m);
}

namespace {

double eta_constant(int m, int d) {
  const double pi = 3.14159265358979323846;
  const int d2 = d / 2;
  if (2 * m <= d) throw std::runtime_error("thin plate spline requires 2m > d");
  double value;
  if (d % 2 == 0) {
    value = ((m + 1 + d2) % 2) ? -1.0 : 1.0;
    for (int i = 0; i < 2 * m - 1; ++i) value /= 2.0;
    for (int i = 0; i < d2; ++i) value /= pi;
    for (int i = 2; i < m; ++i) value /= i;
    for (int i = 2; i <= m - d2; ++i) value /= i;
  } else {
    value = std::sqrt(pi);
    const int k = m - (d - 1) / 2;
    for (int i = 0; i < k; ++i) value /= -0.5 - i;
    for (int i = 0; i < m; ++i) value /= 4.0;
    for (int i = 0; i < d2; ++i) value /= pi;
    value /= std::sqrt(pi);
    for (int i = 2; i < m; ++i) value /= i;
  }
  return value;
}

double eta_r2(int m, int d, double r2, double eta0) {
  if (r2 <= 0.0) return 0.0;
  const int d2 = d / 2;
  double v = eta0;
  if (d % 2 == 0) {
    v *= std::log(r2) * 0.5;
    for (int i = 0; i < m - d2; ++i) v *= r2;
  } else {
    for (int i = 0; i < m - d2 - 1; ++i) v *= r2;
    v *= std::sqrt(r2);
  }
  return v;
}

int default_order(int d) {
  int m = 0;
  while (2 * m < d + 2) ++m;
  return m;
}

int null_space_dimension(int d, int m) {
  int dim = 1;
  for (int i = 0; i < d; ++i) dim *= d + m - 1 - i;
  for (int i = 2; i <= d; ++i) dim /= i;
  return dim;
}

std::vector<int> polynomial_powers(int d, int m, int M) {
  std::vector<int> powers(static_cast<size_t>(M) * d, 0);  // [term * d + coord]
  std::vector<int> index(d, 0);
  for (int term = 0; term < M; ++term) {
    for (int c = 0; c < d; ++c) powers[term * d + c] = index[c];
    int s = 0;
    for (int c = 0; c < d; ++c) s += index[c];
    if (s < m - 1) {
      ++index[0];
    } else {
      s -= index[0];
      index[0] = 0;
      for (int c = 1; c < d; ++c) {
        ++index[c];
        ++s;
        if (s == m) {
          s -= index[c];
          index[c] = 0;
        } else {
          break;
        }
      }
    }
  }
  return powers;
}

// Householder vectors u_t (rows of Z, M x k) with TU H_0 ... H_{M-1} = [0 | L].
std::vector<double> qt_householders(std::vector<double> TU, int M, int k) {
  // TU row-major M x k
  std::vector<double> Z(static_cast<size_t>(M) * k, 0.0);
  for (int step = 0; step < M; ++step) {
    const int L = k - step;
    double* row = &TU[static_cast<size_t>(step) * k];
    double scale = 0.0;
    for (int c = 0; c < L; ++c) scale = std::max(scale, std::fabs(row[c]));
    if (scale != 0.0)
      for (int c = 0; c < L; ++c) row[c] /= scale;
    double length = 0.0;
    for (int c = 0; c < L; ++c) length += row[c] * row[c];
    length = std::sqrt(length);
    if (row[L - 1] < 0.0) length = -length;
    row[L - 1] += length;
    const double mult = length != 0.0 ? 1.0 / (length * row[L - 1]) : 0.0;
    for (int r = step + 1; r < M; ++r) {
      double* other = &TU[static_cast<size_t>(r) * k];
      double proj = 0.0;
      for (int c = 0; c < L; ++c) proj += row[c] * other[c];
      proj *= mult;
      for (int c = 0; c < L; ++c) other[c] -= proj * row[c];
    }
    const double rm = std::sqrt(mult);
    for (int c = 0; c < L; ++c) Z[static_cast<size_t>(step) * k + c] = row[c] * rm;
  }
  return Z;
}

// X (rows x k, column-major) <- X H_0 ... H_{M-1}
void hq_post(std::vector<double>* X, int rows, int k, const std::vector<double>& Z, int M) {
  std::vector<double> prod(rows);
  for (int t = 0; t < M; ++t) {
    const double* u = &Z[static_cast<size_t>(t) * k];
    std::fill(prod.begin(), prod.end(), 0.0);
    for (int c = 0; c < k; ++c)
      for (int r = 0; r < rows; ++r) prod[r] += (*X)[r + static_cast<size_t>(rows) * c] * u[c];
    for (int c = 0; c < k; ++c)
      for (int r = 0; r < rows; ++r) (*X)[r + static_cast<size_t>(rows) * c] -= prod[r] * u[c];
  }
}

// P (k x k) <- H_{M-1} ... H_0 P
void hq_pre_transpose(std::vector<double>* P, int k, const std::vector<double>& Z, int M) {
  std::vector<double> prod(k);
  for (int t = 0; t < M; ++t) {
    const double* u = &Z[static_cast<size_t>(t) * k];
    for (int c = 0; c < k; ++c) {
      double v = 0.0;
      for (int r = 0; r < k; ++r) v += (*P)[r + static_cast<size_t>(k) * c] * u[r];
      prod[c] = v;
    }
    for (int c = 0; c < k; ++c)
      for (int r = 0; r < k; ++r) (*P)[r + static_cast<size_t>(k) * c] -= prod[c] * u[r];
  }
}

}  // namespace

TprsPrep tprs_prepare(const double* cols, int n, int d, int k) {
  const int m = default_order(d);
  const int M = null_space_dimension(d, m);
  std::vector<double> shifted(static_cast<size_t>(n) * d);
  for (int c = 0; c < d; ++c) {
    const double shift = r_mean(cols + static_cast<size_t>(n) * c, n);
    for (int r = 0; r < n; ++r) shifted[r + static_cast<size_t>(n) * c] = cols[r + static_cast<size_t>(n) * c] - shift;
  }
  // sorted unique locations
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    for (int c = 0; c < d; ++c) {
      double va = shifted[a + static_cast<size_t>(n) * c], vb = shifted[b + static_cast<size_t>(n) * c];
      if (va < vb) return true;
      if (va > vb) return false;
    }
    return false;
  });
  std::vector<int> uniq;
  std::vector<int> mapping(n, -1);
  for (int idx : order) {
    bool is_new = uniq.empty();
    if (!is_new) {
      int prior = uniq.back();
      for (int c = 0; c < d; ++c)
        if (shifted[idx + static_cast<size_t>(n) * c] != shifted[prior + static_cast<size_t>(n) * c]) { is_new = true; break; }
    }
    if (is_new) uniq.push_back(idx);
    mapping[idx] = static_cast<int>(uniq.size()) - 1;
  }
  const int nu = static_cast<int>(uniq.size());
  if (nu < k) throw std::runtime_error("thin-plate setup has fewer unique locations than its basis dimension");
  if (nu > 2000) throw std::runtime_error("thin-plate setup supports at most 2000 unique locations");
  std::vector<double> u(static_cast<size_t>(nu) * d);
  for (int i = 0; i < nu; ++i)
    for (int c = 0; c < d; ++c) u[i + static_cast<size_t>(nu) * c] = shifted[uniq[i] + static_cast<size_t>(n) * c];
  std::vector<int> powers = polynomial_powers(d, m, M);
  std::vector<double> T(static_cast<size_t>(nu) * M, 1.0);
  for (int t = 0; t < M; ++t)
    for (int i = 0; i < nu; ++i) {
      double v = 1.0;
      for (int c = 0; c < d; ++c)
        for (int e = 0; e < powers[t * d + c]; ++e) v *= u[i + static_cast<size_t>(nu) * c];
      T[i + static_cast<size_t>(nu) * t] = v;
    }
  TprsPrep prep;
  prep.n = n;
  prep.d = d;
  prep.k = k;
  prep.m = m;
  prep.M = M;
  prep.nu = nu;
  prep.u = std::move(u);
  prep.mapping = std::move(mapping);
  prep.T = std::move(T);
  return prep;
}

double tprs_eta0(int d) { return eta_constant(default_order(d), d); }

std::vector<double> tprs_eta_matrix(const TprsPrep& prep) {
  const int nu = prep.nu, d = prep.d, m = prep.m;
  const std::vector<double>& u = prep.u;
  const double eta0 = eta_constant(m, d);
  std::vector<double> E(static_cast<size_t>(nu) * nu, 0.0);
  for (int j = 0; j < nu; ++j)
    for (int i = 0; i < j; ++i) {
      double r2 = 0.0;
      for (int c = 0; c < d; ++c) {
        double diff = u[i + static_cast<size_t>(nu) * c] - u[j + static_cast<size_t>(nu) * c];
        r2 += diff * diff;
      }
      double v = eta_r2(m, d, r2, eta0);
      E[i + static_cast<size_t>(nu) * j] = v;
      E[j + static_cast<size_t>(nu) * i] = v;
    }
  return E;
}

Smooth tprs_finish(const TprsPrep& prep, const std::vector<double>& vals, const std::vector<double>& U) {
  const int n = prep.n, k = prep.k, M = prep.M, nu = prep.nu;
  const std::vector<double>& T = prep.T;
  const std::vector<int>& mapping = prep.mapping;

  // T'U, row-major M x k
  std::vector<double> TU(static_cast<size_t>(M) * k, 0.0);
  for (int t = 0; t < M; ++t)
    for (int c = 0; c < k; ++c) {
      double s = 0.0;
      for (int i = 0; i < nu; ++i) s += T[i + static_cast<size_t>(nu) * t] * U[i + static_cast<size_t>(nu) * c];
      TU[static_cast<size_t>(t) * k + c] = s;
    }
  std::vector<double> Z = qt_householders(TU, M, k);
  std::vector<double> Xu(static_cast<size_t>(nu) * k);
  for (int c = 0; c < k; ++c)
    for (int i = 0; i < nu; ++i) Xu[i + static_cast<size_t>(nu) * c] = U[i + static_cast<size_t>(nu) * c] * vals[c];
  hq_post(&Xu, nu, k, Z, M);
  for (int t = 0; t < M; ++t)
    for (int i = 0; i < nu; ++i) Xu[i + static_cast<size_t>(nu) * (k - M + t)] = T[i + static_cast<size_t>(nu) * t];
  std::vector<double> X(static_cast<size_t>(n) * k);
  for (int c = 0; c < k; ++c)
    for (int r = 0; r < n; ++r) X[r + static_cast<size_t>(n) * c] = Xu[mapping[r] + static_cast<size_t>(nu) * c];
  std::vector<double> P(static_cast<size_t>(k) * k, 0.0);
  for (int i = 0; i < k; ++i) P[i + static_cast<size_t>(k) * i] = vals[i];
  hq_post(&P, k, k, Z, M);
  hq_pre_transpose(&P, k, Z, M);
  for (int a = 0; a < k; ++a)
    for (int b = k - M; b < k; ++b) {
      P[a + static_cast<size_t>(k) * b] = 0.0;
      P[b + static_cast<size_t>(k) * a] = 0.0;
    }
  for (int c = 0; c < k; ++c) {
    double ss = 0.0;
    for (int r = 0; r < n; ++r) ss += X[r + static_cast<size_t>(n) * c] * X[r + static_cast<size_t>(n) * c];
    double rms = std::sqrt(ss / n);
    if (!std::isfinite(rms) || rms == 0.0) throw std::runtime_error("thin-plate RMS scaling met a zero column");
    for (int r = 0; r < n; ++r) X[r + static_cast<size_t>(n) * c] /= rms;
    for (int i = 0; i < k; ++i) P[c + static_cast<size_t>(k) * i] /= rms;
    for (int i = 0; i < k; ++i) P[i + static_cast<size_t>(k) * c] /= rms;
  }
  std::vector<double> Ps(static_cast<size_t>(k) * k);
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b)
      Ps[a + static_cast<size_t>(k) * b] = (P[a + static_cast<size_t>(k) * b] + P[b + static_cast<size_t>(k) * a]) / 2.0;
  double xnorm = 0.0;
  for (int r = 0; r < n; ++r) {
    double s = 0.0;
    for (int c = 0; c < k; ++c) s += std::fabs(X[r + static_cast<size_t>(n) * c]);
    xnorm = std::max(xnorm, s);
  }
  double pnorm = 0.0;
  for (int c = 0; c < k; ++c) {
    double s = 0.0;
    for (int a = 0; a < k; ++a) s += std::fabs(Ps[a + static_cast<size_t>(k) * c]);
    pnorm = std::max(pnorm, s);
  }
  const double pscale = pnorm / (xnorm * xnorm);
  if (!std::isfinite(pscale) || pscale <= 0.0) throw std::runtime_error("thin-plate penalty scaling failed");
  for (double& v : Ps) v /= pscale;
  // centering constraint: Householder H = I - v v'/v0 of colMeans(X)
  std::vector<double> cm(k);
  for (int c = 0; c < k; ++c) cm[c] = r_mean(&X[static_cast<size_t>(n) * c], n);
  double nrm = 0.0;
  for (double v : cm) nrm += v * v;
  nrm = std::sqrt(nrm);
  if (nrm == 0.0) throw std::runtime_error("centering constraint is rank deficient");
  if (cm[0] != 0.0) nrm = std::copysign(nrm, cm[0]);
  std::vector<double> hv(k);
  for (int c = 0; c < k; ++c) hv[c] = cm[c] / nrm;
  hv[0] += 1.0;
  const double v0 = hv[0];
  // XH: each row x -> x - (x.v / v0) v
  Smooth out;
  out.n = n;
  out.cols = k - 1;
  out.rank = k - M;
  out.X.assign(static_cast<size_t>(n) * (k - 1), 0.0);
  for (int r = 0; r < n; ++r) {
    double dv = 0.0;
    for (int c = 0; c < k; ++c) dv += X[r + static_cast<size_t>(n) * c] * hv[c];
    dv /= v0;
    for (int c = 1; c < k; ++c) out.X[r + static_cast<size_t>(n) * (c - 1)] = X[r + static_cast<size_t>(n) * c] - dv * hv[c];
  }
  // H S H
  std::vector<double> HS(static_cast<size_t>(k) * k);
  for (int c = 0; c < k; ++c) {
    double dv = 0.0;
    for (int a = 0; a < k; ++a) dv += hv[a] * Ps[a + static_cast<size_t>(k) * c];
    dv /= v0;
    for (int a = 0; a < k; ++a) HS[a + static_cast<size_t>(k) * c] = Ps[a + static_cast<size_t>(k) * c] - dv * hv[a];
  }
  out.S.assign(static_cast<size_t>(k - 1) * (k - 1), 0.0);
  for (int a = 0; a < k; ++a) {
    double dv = 0.0;
    for (int c = 0; c < k; ++c) dv += HS[a + static_cast<size_t>(k) * c] * hv[c];
    dv /= v0;
    if (a == 0) continue;
    for (int c = 1; c < k; ++c)
      out.S[(a - 1) + static_cast<size_t>(k - 1) * (c - 1)] = HS[a + static_cast<size_t>(k) * c] - dv * hv[c];
  }
  return out;
}

Smooth build_smooth(const double* cols, int n, int d, int k) {
  TprsPrep prep = tprs_prepare(cols, n, d, k);
  std::vector<double> E = tprs_eta_matrix(prep);
  std::vector<double> vals, U;
  top_magnitude_eigen(E.data(), prep.nu, k, &vals, &U);
  return tprs_finish(prep, vals, U);
}

// Sum of squares of each column of an n x cols matrix, accumulated in long
// double in row order.
std::vector<double> column_sumsq(const double* X, int n, int cols) {
  std::vector<double> out(cols);
  for (int c = 0; c < cols; ++c) {
    long double t = 0.0L;
    for (int r = 0; r < n; ++r) {
      double v = X[r + static_cast<size_t>(n) * c];
      t += v * v;
    }
    out[c] = static_cast<double>(t);
  }
  return out;
}

std::vector<double> initial_sp(const Design& des) {
  return initial_sp_from_colsq(des, column_sumsq(des.X.data(), des.n, des.q));
}

std::vector<double> initial_sp_from_colsq(const Design& des, const std::vector<double>& xdiag) {
  const int q = des.q;
  std::vector<double> pdiag(q, 0.0);
  std::vector<char> penalized(q, 0);
  const double thr_scale = std::pow(2.220446049250313e-16, 0.8);
  std::vector<double> result(des.m);
  for (int j = 0; j < des.m; ++j) {
    const int dim = des.dims[j], off = des.offsets[j];
    const std::vector<double>& S = des.blocks[j];
    double mx = 0.0;
    for (double v : S) mx = std::max(mx, std::fabs(v));
    const double thr = thr_scale * mx;
    std::vector<double> ax, ap;
    std::vector<int> active;
    std::vector<double> rowabs(dim), colabs(dim);
    for (int c = 0; c < dim; ++c) {
      for (int o = 0; o < dim; ++o) {
        rowabs[o] = std::fabs(S[c + static_cast<size_t>(dim) * o]);
        colabs[o] = std::fabs(S[o + static_cast<size_t>(dim) * c]);
      }
      double rm = r_mean(rowabs.data(), dim), cmn = r_mean(colabs.data(), dim);
      double dg = std::fabs(S[c + static_cast<size_t>(dim) * c]);
      if (rm > thr && cmn > thr && dg > thr) {
        active.push_back(c);
        ax.push_back(xdiag[off + c]);
        ap.push_back(S[c + static_cast<size_t>(dim) * c]);
      }
    }
    if (active.empty()) throw std::runtime_error("initial.sp found no active coordinates");
    double lam = r_mean(ax.data(), static_cast<int>(ax.size())) / r_mean(ap.data(), static_cast<int>(ap.size()));
    result[j] = lam;
    for (int c : active) penalized[off + c] = 1;
    for (int c = 0; c < dim; ++c) pdiag[off + c] += lam * S[c + static_cast<size_t>(dim) * c];
  }
  std::vector<int> used;
  for (int c = 0; c < q; ++c)
    if (pdiag[c] > 0.0 && penalized[c] && xdiag[c] > 0.0) used.push_back(c);
  if (used.empty()) throw std::runtime_error("initial.sp has no used coordinates");
  auto mean_hat = [&]() {
    std::vector<double> h;
    for (int c : used) h.push_back(xdiag[c] / (xdiag[c] + pdiag[c]));
    return r_mean(h.data(), static_cast<int>(h.size()));
  };
  int guard = 0;
  while (mean_hat() > 0.4) {
    for (double& v : result) v *= 10.0;
    for (double& v : pdiag) v *= 10.0;
    if (++guard > 1000) throw std::runtime_error("initial.sp did not bracket 0.4");
  }
  while (mean_hat() < 0.4) {
    for (double& v : result) v /= 10.0;
    for (double& v : pdiag) v /= 10.0;
    if (++guard > 2000) throw std::runtime_error("initial.sp did not bracket 0.4");
  }
  return result;
}

void prepare_geometry(Design* des) {
  const int n = des->n, q = des->q;
  householder_qr(des->X.data(), n, q, &des->Q, &des->R);
  for (int c = 0; c < q; ++c)
    if (des->R[c + static_cast<size_t>(q) * c] == 0.0) throw std::runtime_error("design matrix is rank deficient");
  if (des->m == 1) {
    // Ri = R^-1 (upper triangular)
    std::vector<double> Ri(static_cast<size_t>(q) * q, 0.0);
    for (int c = 0; c < q; ++c) {
      Ri[c + static_cast<size_t>(q) * c] = 1.0 / des->R[c + static_cast<size_t>(q) * c];
      for (int r = c - 1; r >= 0; --r) {
        double s = 0.0;
        for (int t = r + 1; t <= c; ++t) s += des->R[r + static_cast<size_t>(q) * t] * Ri[t + static_cast<size_t>(q) * c];
        Ri[r + static_cast<size_t>(q) * c] = -s / des->R[r + static_cast<size_t>(q) * r];
      }
    }
    std::vector<double> Sf(static_cast<size_t>(q) * q, 0.0);
    const int off = des->offsets[0], dim = des->dims[0];
    for (int b = 0; b < dim; ++b)
      for (int a = 0; a < dim; ++a) Sf[(off + a) + static_cast<size_t>(q) * (off + b)] = des->blocks[0][a + static_cast<size_t>(dim) * b];
    std::vector<double> SRi(static_cast<size_t>(q) * q, 0.0), Wm(static_cast<size_t>(q) * q, 0.0);
    for (int c = 0; c < q; ++c)
      for (int t = 0; t < q; ++t) {
        double v = Ri[t + static_cast<size_t>(q) * c];
        if (v == 0.0) continue;
        for (int r = 0; r < q; ++r) SRi[r + static_cast<size_t>(q) * c] += Sf[r + static_cast<size_t>(q) * t] * v;
      }
    for (int c = 0; c < q; ++c)
      for (int r = 0; r < q; ++r) {
        double s = 0.0;
        for (int t = 0; t < q; ++t) s += Ri[t + static_cast<size_t>(q) * r] * SRi[t + static_cast<size_t>(q) * c];
        Wm[r + static_cast<size_t>(q) * c] = s;
      }
    for (int c = 0; c < q; ++c)
      for (int r = c + 1; r < q; ++r) {
        double s = 0.5 * (Wm[r + static_cast<size_t>(q) * c] + Wm[c + static_cast<size_t>(q) * r]);
        Wm[r + static_cast<size_t>(q) * c] = Wm[c + static_cast<size_t>(q) * r] = s;
      }
    std::vector<double> vals, vecs;
    jacobi_eigen(Wm.data(), q, &vals, &vecs);
    des->spec.assign(q, 0.0);
    std::vector<double> V(static_cast<size_t>(q) * q);
    for (int c = 0; c < q; ++c) {
      const int src = q - 1 - c;
      des->spec[c] = c < des->ranks[0] ? std::max(0.0, vals[src]) : 0.0;
      for (int r = 0; r < q; ++r) V[r + static_cast<size_t>(q) * c] = vecs[r + static_cast<size_t>(q) * src];
    }
    des->QW.assign(static_cast<size_t>(n) * q, 0.0);
    for (int c = 0; c < q; ++c)
      for (int t = 0; t < q; ++t) {
        double v = V[t + static_cast<size_t>(q) * c];
        const double* qt = &des->Q[static_cast<size_t>(n) * t];
        double* out = &des->QW[static_cast<size_t>(n) * c];
        for (int r = 0; r < n; ++r) out[r] += qt[r] * v;
      }
  } else {
    des->roots.clear();
    for (int j = 0; j < des->m; ++j) des->roots.push_back(penalty_root(des->blocks[j], des->dims[j], des->ranks[j]));
  }
}

std::vector<double> penalty_root(const std::vector<double>& block, int dim, int rank) {
  std::vector<double> S = block;
  for (int c = 0; c < dim; ++c)
    for (int r = c + 1; r < dim; ++r) {
      double s = 0.5 * (S[r + static_cast<size_t>(dim) * c] + S[c + static_cast<size_t>(dim) * r]);
      S[r + static_cast<size_t>(dim) * c] = S[c + static_cast<size_t>(dim) * r] = s;
    }
  std::vector<double> vals, vecs;
  jacobi_eigen(S.data(), dim, &vals, &vecs);
  std::vector<double> root(static_cast<size_t>(dim) * rank);
  for (int c = 0; c < rank; ++c) {
    const int src = dim - 1 - c;
    const double s = std::sqrt(std::max(0.0, vals[src]));
    for (int r = 0; r < dim; ++r) root[r + static_cast<size_t>(dim) * c] = vecs[r + static_cast<size_t>(dim) * src] * s;
  }
  return root;
}

std::shared_ptr<Design> build_additive_meta(int n, int p, const std::vector<int>& S, DesignCache* cache) {
  if (S.size() < 3) throw std::runtime_error("an additive design needs |S| >= 3");
  for (int s : S)
    if (s < 0 || s >= p) throw std::runtime_error("conditioning index out of range");
  auto des = std::make_shared<Design>();
  des->n = n;
  des->S = S;
  des->device_geometry = true;
  for (int s : S) des->parts.push_back(cache->univariate(s));
  int q = 1;
  for (auto& sm : des->parts) q += sm->cols;
  if (q >= n) throw std::runtime_error("design width must be below n");
  des->q = q;
  des->m = static_cast<int>(des->parts.size());
  // the intercept column's sum of squares is n, exactly as accumulated
  std::vector<double> xdiag(1, column_sumsq(std::vector<double>(n, 1.0).data(), n, 1)[0]);
  int dest = 1;
  for (auto& sm : des->parts) {
    des->blocks.push_back(sm->S);
    des->offsets.push_back(dest);
    des->dims.push_back(sm->cols);
    des->ranks.push_back(sm->rank);
    des->roots.push_back(sm->root);
    xdiag.insert(xdiag.end(), sm->colsq.begin(), sm->colsq.end());
    dest += sm->cols;
  }
  std::vector<double> sp = initial_sp_from_colsq(*des, xdiag);
  des->initial_log_sp.resize(sp.size());
  for (size_t j = 0; j < sp.size(); ++j) des->initial_log_sp[j] = std::log(sp[j]);
  return des;
}

std::shared_ptr<Design> build_design(const double* data, int n, int p, const std::vector<int>& S,
                                     DesignCache* cache) {
  if (S.empty()) throw std::runtime_error("an empty conditioning set has no design");
  for (int s : S)
    if (s < 0 || s >= p) throw std::runtime_error("conditioning index out of range");
  auto des = std::make_shared<Design>();
  des->n = n;
  des->S = S;
  std::vector<std::shared_ptr<const Smooth>> parts;
  if (S.size() <= 2) {
    std::vector<double> cols(static_cast<size_t>(n) * S.size());
    for (size_t c = 0; c < S.size(); ++c)
      std::copy(data + static_cast<size_t>(n) * S[c], data + static_cast<size_t>(n) * (S[c] + 1), cols.begin() + static_cast<size_t>(n) * c);
    std::shared_ptr<const Smooth> pre = (S.size() == 2 && cache) ? cache->bivariate(S) : nullptr;
    if (S.size() == 1 && cache) {
      parts.push_back(cache->univariate(S[0]));
    } else if (pre) {
      parts.push_back(pre);
    } else {
      parts.push_back(std::make_shared<Smooth>(build_smooth(cols.data(), n, static_cast<int>(S.size()), S.size() == 1 ? 10 : 30)));
    }
  } else {
    for (int s : S) {
      if (cache) parts.push_back(cache->univariate(s));
      else parts.push_back(std::make_shared<Smooth>(build_smooth(data + static_cast<size_t>(n) * s, n, 1, 10)));
    }
  }
  int q = 1;
  for (auto& sm : parts) q += sm->cols;
  if (q >= n) throw std::runtime_error("design width must be below n");
  des->q = q;
  des->m = static_cast<int>(parts.size());
  des->X.assign(static_cast<size_t>(n) * q, 0.0);
  for (int r = 0; r < n; ++r) des->X[r] = 1.0;
  int dest = 1;
  for (auto& sm : parts) {
    std::copy(sm->X.begin(), sm->X.end(), des->X.begin() + static_cast<size_t>(n) * dest);
    des->blocks.push_back(sm->S);
    des->offsets.push_back(dest);
    des->dims.push_back(sm->cols);
    des->ranks.push_back(sm->rank);
    dest += sm->cols;
  }
  std::vector<double> sp = initial_sp(*des);
  des->initial_log_sp.resize(sp.size());
  for (size_t j = 0; j < sp.size(); ++j) des->initial_log_sp[j] = std::log(sp[j]);
  prepare_geometry(des.get());
  return des;
}

std::shared_ptr<Design> build_single_meta(int n, int p, const std::vector<int>& S, DesignCache* cache) {
  if (S.empty() || S.size() > 2) throw std::runtime_error("a single-penalty design needs |S| of 1 or 2");
  for (int s : S)
    if (s < 0 || s >= p) throw std::runtime_error("conditioning index out of range");
  std::shared_ptr<const Smooth> sm;
  if (S.size() == 1) {
    sm = cache->univariate(S[0]);
  } else {
    sm = cache->bivariate(S);
    if (!sm) {
      std::vector<double> cols(static_cast<size_t>(n) * 2);
      for (size_t c = 0; c < 2; ++c)
        std::copy(cache->data() + static_cast<size_t>(n) * S[c], cache->data() + static_cast<size_t>(n) * (S[c] + 1),
                  cols.begin() + static_cast<size_t>(n) * c);
      auto built = std::make_shared<Smooth>(build_smooth(cols.data(), n, 2, 30));
      built->colsq = column_sumsq(built->X.data(), built->n, built->cols);
      sm = built;
    }
  }
  auto des = std::make_shared<Design>();
  des->n = n;
  des->S = S;
  des->device_geometry = true;
  des->q = 1 + sm->cols;
  if (des->q >= n) throw std::runtime_error("design width must be below n");
  des->m = 1;
  des->blocks.push_back(sm->S);
  des->offsets.push_back(1);
  des->dims.push_back(sm->cols);
  des->ranks.push_back(sm->rank);
  std::vector<double> xdiag(1, column_sumsq(std::vector<double>(n, 1.0).data(), n, 1)[0]);
  std::vector<double> colsq = sm->colsq.empty() ? column_sumsq(sm->X.data(), sm->n, sm->cols) : sm->colsq;
  xdiag.insert(xdiag.end(), colsq.begin(), colsq.end());
  std::vector<double> sp = initial_sp_from_colsq(*des, xdiag);
  des->initial_log_sp.assign(1, std::log(sp[0]));
  des->parts.push_back(sm);
  return des;
}

std::shared_ptr<const Smooth> DesignCache::univariate(int column) {
  {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = uni_.find(column);
    if (it != uni_.end()) return it->second;
  }
  auto built = std::make_shared<Smooth>(build_smooth(data_ + static_cast<size_t>(n_) * column, n_, 1, 10));
  built->colsq = column_sumsq(built->X.data(), built->n, built->cols);
  built->root = penalty_root(built->S, built->cols, built->rank);
  std::shared_ptr<const Smooth> sm = built;
  std::lock_guard<std::mutex> lock(mu_);
  auto it = uni_.find(column);
  if (it != uni_.end()) return it->second;
  uni_[column] = sm;
  return sm;
}

void DesignCache::put_univariate(int column, std::shared_ptr<const Smooth> smooth) {
  std::lock_guard<std::mutex> lock(mu_);
  uni_[column] = std::move(smooth);
}

bool DesignCache::has_univariate(int column) {
  std::lock_guard<std::mutex> lock(mu_);
  return uni_.count(column) > 0;
}

void DesignCache::put_bivariate(const std::vector<int>& S, std::shared_ptr<const Smooth> smooth) {
  std::lock_guard<std::mutex> lock(mu_);
  bi_[S] = std::move(smooth);
}

std::shared_ptr<const Smooth> DesignCache::bivariate(const std::vector<int>& S) {
  std::lock_guard<std::mutex> lock(mu_);
  auto it = bi_.find(S);
  return it == bi_.end() ? nullptr : it->second;
}

bool DesignCache::has_design(const std::vector<int>& S) {
  std::lock_guard<std::mutex> lock(mu_);
  return designs_.count(S) > 0 || bi_.count(S) > 0;
}

std::vector<std::shared_ptr<const Design>> DesignCache::find_designs(const std::vector<const std::vector<int>*>& sets) {
  std::vector<std::shared_ptr<const Design>> out(sets.size());
  std::lock_guard<std::mutex> lock(mu_);
  for (size_t i = 0; i < sets.size(); ++i) {
    auto it = designs_.find(*sets[i]);
    if (it != designs_.end()) out[i] = it->second;
  }
  return out;
}

std::shared_ptr<const Design> DesignCache::build(const std::vector<int>& S) {
  return S.size() >= 3 ? build_additive_meta(n_, p_, S, this) : build_single_meta(n_, p_, S, this);
}

void DesignCache::put_designs(const std::vector<const std::vector<int>*>& sets,
                              const std::vector<std::shared_ptr<const Design>>& designs) {
  std::lock_guard<std::mutex> lock(mu_);
  for (size_t i = 0; i < sets.size(); ++i)
    if (designs[i]) designs_.emplace(*sets[i], designs[i]);
}

std::shared_ptr<const Design> DesignCache::get(const std::vector<int>& S) {
  {
    std::lock_guard<std::mutex> lock(mu_);
    auto it = designs_.find(S);
    if (it != designs_.end()) return it->second;
  }
  std::shared_ptr<const Design> d =
      S.size() >= 3 ? build_additive_meta(n_, p_, S, this) : build_single_meta(n_, p_, S, this);
  std::lock_guard<std::mutex> lock(mu_);
  auto it = designs_.find(S);
  if (it != designs_.end()) return it->second;
  designs_[S] = d;
  return d;
}

}  // namespace fkpc
