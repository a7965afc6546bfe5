#include "hostla.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <stdexcept>

namespace fkpc {

namespace {

// Dot product with eight independent partial sums: the chains overlap and
// the compiler vectorises them without reassociation flags.
__attribute__((always_inline)) inline double dot_chains(const double* a, const double* b, int len) {
  double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int i = 0;
  for (; i + 8 <= len; i += 8)
    for (int t = 0; t < 8; ++t) s[t] += a[i + t] * b[i + t];
  double tail = 0.0;
  for (; i < len; ++i) tail += a[i] * b[i];
  return (((s[0] + s[4]) + (s[1] + s[5])) + ((s[2] + s[6]) + (s[3] + s[7]))) + tail;
}

// Householder QR, Q formed explicitly by backward accumulation.  When H_k is
// applied to the columns of the (partial) Q, columns j < k are still e_j,
// which H_k leaves alone, so only columns k.. are touched.
__attribute__((always_inline)) inline void householder_qr_core(const double* A, int rows, int cols,
                                                              std::vector<double>* Q, std::vector<double>* R) {
  std::vector<double> W(A, A + static_cast<size_t>(rows) * cols);
  std::vector<double> V(static_cast<size_t>(rows) * cols, 0.0);
  std::vector<double> beta(cols, 0.0);
  for (int k = 0; k < cols; ++k) {
    double* x = &W[static_cast<size_t>(k) * rows];
    const int len = rows - k;
    const double norm2 = dot_chains(x + k, x + k, len);
    const double norm = std::sqrt(norm2);
    double* v = &V[static_cast<size_t>(k) * rows];
    if (norm == 0.0) { beta[k] = 0.0; continue; }
    const double alpha = x[k] >= 0.0 ? -norm : norm;
    for (int i = k; i < rows; ++i) v[i] = x[i];
    v[k] -= alpha;
    const double vnorm2 = norm2 - x[k] * x[k] + v[k] * v[k];
    beta[k] = 2.0 / vnorm2;
    // apply H = I - beta v v' to columns k..cols-1
    for (int j = k; j < cols; ++j) {
      double* c = &W[static_cast<size_t>(j) * rows];
      const double dot = dot_chains(v + k, c + k, len) * beta[k];
      for (int i = k; i < rows; ++i) c[i] -= dot * v[i];
    }
  }
  R->assign(static_cast<size_t>(cols) * cols, 0.0);
  for (int j = 0; j < cols; ++j)
    for (int i = 0; i <= j; ++i) (*R)[i + static_cast<size_t>(cols) * j] = W[i + static_cast<size_t>(rows) * j];
  Q->assign(static_cast<size_t>(rows) * cols, 0.0);
  for (int j = 0; j < cols; ++j) (*Q)[j + static_cast<size_t>(rows) * j] = 1.0;
  for (int k = cols - 1; k >= 0; --k) {
    if (beta[k] == 0.0) continue;
    const double* v = &V[static_cast<size_t>(k) * rows];
    const int len = rows - k;
    for (int j = k; j < cols; ++j) {
      double* c = &(*Q)[static_cast<size_t>(j) * rows];
      const double dot = dot_chains(v + k, c + k, len) * beta[k];
      for (int i = k; i < rows; ++i) c[i] -= dot * v[i];
    }
  }
}

__attribute__((target("avx2,fma"))) void householder_qr_avx2(const double* A, int rows, int cols,
                                                             std::vector<double>* Q, std::vector<double>* R) {
  householder_qr_core(A, rows, cols, Q, R);
}

void householder_qr_generic(const double* A, int rows, int cols, std::vector<double>* Q, std::vector<double>* R) {
  householder_qr_core(A, rows, cols, Q, R);
}

}  // namespace

// The AVX2/FMA build of the same loops where the host CPU has them, chosen
// once per process, so every design of a process is factored the same way.
void householder_qr(const double* A, int rows, int cols, std::vector<double>* Q,
                    std::vector<double>* R) {
  if (rows < cols || cols <= 0) throw std::runtime_error("householder_qr: need rows >= cols > 0");
  static const bool avx2 = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
  if (avx2) householder_qr_avx2(A, rows, cols, Q, R);
  else householder_qr_generic(A, rows, cols, Q, R);
}

void jacobi_eigen(const double* A, int n, std::vector<double>* values,
                  std::vector<double>* vectors) {
  std::vector<double> a(A, A + static_cast<size_t>(n) * n);
  std::vector<double> v(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) v[i + static_cast<size_t>(n) * i] = 1.0;
  auto at = [&](int i, int j) -> double& { return a[i + static_cast<size_t>(n) * j]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        if (i == j) diag += at(i, i) * at(i, i);
        else off += at(i, j) * at(i, j);
      }
    if (off <= 1e-32 * diag || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        double apq = at(p, q);
        if (apq == 0.0) continue;
        double app = at(p, p), aqq = at(q, q);
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0);
        double s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = at(k, p), akq = at(k, q);
          at(k, p) = c * akp - s * akq;
          at(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = at(p, k), aqk = at(q, k);
          at(p, k) = c * apk - s * aqk;
          at(q, k) = s * apk + c * aqk;
        }
        at(p, q) = 0.0;
        at(q, p) = 0.0;
        for (int k = 0; k < n; ++k) {
          double vkp = v[k + static_cast<size_t>(n) * p], vkq = v[k + static_cast<size_t>(n) * q];
          v[k + static_cast<size_t>(n) * p] = c * vkp - s * vkq;
          v[k + static_cast<size_t>(n) * q] = s * vkp + c * vkq;
        }
      }
    }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int l, int r) { return at(l, l) < at(r, r); });
  values->resize(n);
  vectors->resize(static_cast<size_t>(n) * n);
  for (int j = 0; j < n; ++j) {
    (*values)[j] = at(order[j], order[j]);
    for (int i = 0; i < n; ++i)
      (*vectors)[i + static_cast<size_t>(n) * j] = v[i + static_cast<size_t>(n) * order[j]];
  }
}

bool tridiagonal_ql(int n, double* d, double* e, double* z) {
  if (n <= 0) return true;
  e[n - 1] = 0.0;
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) return false;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      for (; i >= l; --i) {
        double f = s * e[i];
        double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          double zk1 = z[k + static_cast<size_t>(n) * (i + 1)];
          double zk = z[k + static_cast<size_t>(n) * i];
          z[k + static_cast<size_t>(n) * (i + 1)] = s * zk + c * zk1;
          z[k + static_cast<size_t>(n) * i] = c * zk - s * zk1;
        }
      }
      if (r == 0.0 && i >= l) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return true;
}

namespace {

__attribute__((always_inline)) inline void symv(const double* A, int n, const double* x, double* y) {
  // upper triangle only: column j gives y[i] += A(i,j) x[j] and y[j] += A(i,j) x[i], i < j
  for (int i = 0; i < n; ++i) y[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    const double xj = x[j];
    const double* col = A + static_cast<size_t>(n) * j;
    double s0 = 0.0, s1 = 0.0;
    int i = 0;
    for (; i + 1 < j; i += 2) {
      y[i] += col[i] * xj;
      y[i + 1] += col[i + 1] * xj;
      s0 += col[i] * x[i];
      s1 += col[i + 1] * x[i + 1];
    }
    for (; i < j; ++i) {
      y[i] += col[i] * xj;
      s0 += col[i] * x[i];
    }
    y[j] += (s0 + s1) + col[j] * xj;
  }
}

__attribute__((always_inline)) inline double dot(const double* a, const double* b, int n) {
  return dot_chains(a, b, n);
}

// indices of the k entries of largest |value| (ties toward the lower index)
std::vector<int> top_k_by_magnitude(const std::vector<double>& v, int count, int k) {
  std::vector<int> idx(count);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return std::fabs(v[a]) > std::fabs(v[b]); });
  idx.resize(k);
  return idx;
}

}  // namespace

int top_magnitude_eigen(const double* A, int n, int k, std::vector<double>* values,
                        std::vector<double>* vectors) {
  if (k <= 0 || k > n) throw std::runtime_error("top_magnitude_eigen: invalid k");
  const int maxit = n;
  std::vector<double> Qv(static_cast<size_t>(n) * (maxit + 1), 0.0);
  std::vector<double> alpha(maxit + 1, 0.0), beta(maxit + 1, 0.0);
  // deterministic start vector from a small LCG
  unsigned long state = 1;
  double norm = 0.0;
  for (int i = 0; i < n; ++i) {
    state = (state * 106UL + 1283UL) % 6075UL;
    Qv[i] = static_cast<double>(state) / 6075.0 - 0.5;
    norm += Qv[i] * Qv[i];
  }
  norm = std::sqrt(norm);
  for (int i = 0; i < n; ++i) Qv[i] /= norm;
  std::vector<double> w(n), theta, S, dwork, ework;
  uint64_t restart_seed = 0x5eedu;
  int steps = 0;
  const double tol = 1e-14;
  double anorm = 0.0;
  for (int j = 0; j < maxit; ++j) {
    double* qj = &Qv[static_cast<size_t>(n) * j];
    symv(A, n, qj, w.data());
    alpha[j] = dot(qj, w.data(), n);
    for (int i = 0; i < n; ++i) w[i] -= alpha[j] * qj[i];
    if (j > 0) {
      const double* qp = &Qv[static_cast<size_t>(n) * (j - 1)];
      for (int i = 0; i < n; ++i) w[i] -= beta[j - 1] * qp[i];
    }
    for (int pass = 0; pass < 2; ++pass) {
      for (int b = 0; b <= j; ++b) {
        const double* qb = &Qv[static_cast<size_t>(n) * b];
        double c = dot(w.data(), qb, n);
        for (int i = 0; i < n; ++i) w[i] -= c * qb[i];
      }
    }
    beta[j] = std::sqrt(dot(w.data(), w.data(), n));
    steps = j + 1;
    anorm = std::max(anorm, std::fabs(alpha[j]) + beta[j] + (j > 0 ? beta[j - 1] : 0.0));
    bool invariant = beta[j] <= 1e-15 * anorm;
    bool check = invariant || j + 1 == maxit || (j + 1 >= k + 5 && ((j + 1 - k) % 5 == 0));
    if (check) {
      int m = j + 1;
      dwork.assign(alpha.begin(), alpha.begin() + m);
      ework.assign(m, 0.0);
      for (int i = 0; i + 1 < m; ++i) ework[i] = beta[i];
      S.assign(static_cast<size_t>(m) * m, 0.0);
      for (int i = 0; i < m; ++i) S[i + static_cast<size_t>(m) * i] = 1.0;
      if (!tridiagonal_ql(m, dwork.data(), ework.data(), S.data()))
        throw std::runtime_error("Lanczos tridiagonal eigen-solve failed");
      std::vector<int> sel = top_k_by_magnitude(dwork, m, std::min(k, m));
      double tmax = 0.0;
      for (int i = 0; i < m; ++i) tmax = std::max(tmax, std::fabs(dwork[i]));
      bool converged = m >= k;
      if (converged && !invariant) {
        for (int i : sel) {
          double resid = std::fabs(beta[j] * S[(m - 1) + static_cast<size_t>(m) * i]);
          if (resid > tol * tmax) { converged = false; break; }
        }
      }
      // an invariant subspace smaller than k (many near-duplicate locations
      // make the matrix numerically rank deficient): restart below instead
      const bool restart = invariant && m < k && j + 1 < maxit;
      if (!restart && (converged || invariant || j + 1 == maxit)) {
        if (m < k) throw std::runtime_error("Lanczos produced fewer Ritz pairs than requested");
        theta.assign(k, 0.0);
        std::vector<double> V(static_cast<size_t>(n) * k, 0.0);
        for (int c = 0; c < k; ++c) {
          int i = sel[c];
          theta[c] = dwork[i];
          for (int b = 0; b < m; ++b) {
            double coef = S[b + static_cast<size_t>(m) * i];
            const double* qb = &Qv[static_cast<size_t>(n) * b];
            double* vc = &V[static_cast<size_t>(n) * c];
            for (int r = 0; r < n; ++r) vc[r] += coef * qb[r];
          }
        }
        // Rayleigh-Ritz within span(V): H = V'AV, with AV as one pass over A
        // (column j of A updates every column of AV), then rotate V.
        std::vector<double> AV(static_cast<size_t>(n) * k, 0.0);
        for (int jj = 0; jj < n; ++jj) {
          const double* acol = A + static_cast<size_t>(n) * jj;
          for (int c = 0; c < k; ++c) {
            const double vjc = V[jj + static_cast<size_t>(n) * c];
            double* avc = &AV[static_cast<size_t>(n) * c];
            for (int i = 0; i < n; ++i) avc[i] += acol[i] * vjc;
          }
        }
        std::vector<double> H(static_cast<size_t>(k) * k);
        for (int a = 0; a < k; ++a)
          for (int b = 0; b <= a; ++b) {
            const double h = 0.5 * (dot(&V[static_cast<size_t>(n) * a], &AV[static_cast<size_t>(n) * b], n) +
                                    dot(&V[static_cast<size_t>(n) * b], &AV[static_cast<size_t>(n) * a], n));
            H[a + static_cast<size_t>(k) * b] = H[b + static_cast<size_t>(k) * a] = h;
          }
        std::vector<double> hv, hz;
        jacobi_eigen(H.data(), k, &hv, &hz);
        std::vector<int> pick(k);
        for (int c = 0; c < k; ++c) pick[c] = c;
        std::stable_sort(pick.begin(), pick.end(), [&](int a, int b) { return hv[a] > hv[b]; });
        values->assign(k, 0.0);
        vectors->assign(static_cast<size_t>(n) * k, 0.0);
        for (int c = 0; c < k; ++c) {
          int i = pick[c];
          (*values)[c] = hv[i];
          double* out = &(*vectors)[static_cast<size_t>(n) * c];
          for (int b = 0; b < k; ++b) {
            double coef = hz[b + static_cast<size_t>(k) * i];
            const double* vb = &V[static_cast<size_t>(n) * b];
            for (int r = 0; r < n; ++r) out[r] += coef * vb[r];
          }
          double nn = std::sqrt(dot(out, out, n));
          int imax = 0;
          double amax = -1.0;
          for (int r = 0; r < n; ++r) {
            out[r] /= nn;
            if (std::fabs(out[r]) > amax) { amax = std::fabs(out[r]); imax = r; }
          }
          if (out[imax] < 0.0)
            for (int r = 0; r < n; ++r) out[r] = -out[r];
        }
        return steps;
      }
    }
    double* qn = &Qv[static_cast<size_t>(n) * (j + 1)];
    if (invariant) {
      // Deflated restart: the Krylov space is invariant, so the tridiagonal
      // splits here (beta = 0) and the iteration goes on from a new start
      // vector orthogonal to every Lanczos vector so far.  The pairs found
      // after it belong to the rest of the spectrum (near zero when the
      // split came from near-duplicate locations).
      beta[j] = 0.0;
      double nn = 0.0;
      for (int attempt = 0; attempt < 8 && !(nn > 1e-8); ++attempt) {
        for (int i = 0; i < n; ++i) {  // splitmix64 stream, seeded by the step
          uint64_t z = (restart_seed += 0x9e3779b97f4a7c15ull);
          z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
          z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
          z ^= z >> 31;
          qn[i] = static_cast<double>(z >> 11) * 0x1.0p-53 - 0.5;
        }
        for (int pass = 0; pass < 2; ++pass)
          for (int b = 0; b <= j; ++b) {
            const double* qb = &Qv[static_cast<size_t>(n) * b];
            const double c = dot(qn, qb, n);
            for (int i = 0; i < n; ++i) qn[i] -= c * qb[i];
          }
        nn = std::sqrt(dot(qn, qn, n)) / std::sqrt(static_cast<double>(n));
      }
      if (!(nn > 1e-8)) throw std::runtime_error("Lanczos restart found no new direction");
      const double inv = 1.0 / (nn * std::sqrt(static_cast<double>(n)));
      for (int i = 0; i < n; ++i) qn[i] *= inv;
      continue;
    }
    for (int i = 0; i < n; ++i) qn[i] = w[i] / beta[j];
  }
  throw std::runtime_error("Lanczos did not converge");
}


}  // namespace fkpc
