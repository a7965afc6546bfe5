// regrXonS design setup: mgcv-style thin-plate (|S| <= 2) and additive
// (|S| > 2) smooth bases, penalties, initial smoothing parameters and the
// per-design geometry the GPU fit kernels consume.
#pragma once
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace fkpc {

struct Smooth {
  int n = 0, cols = 0, rank = 0;   // cols = k - 1 after the centering constraint
  std::vector<double> X;           // n x cols, column-major
  std::vector<double> S;           // cols x cols penalty
  // univariate smooths of the design cache only: what every additive design
  // containing the variable reuses
  std::vector<double> colsq;       // cols: sum of squares of each column of X
  std::vector<double> root;        // cols x rank: root root' = S
  // bivariate smooths built on the device: X lives in device memory owned by
  // the engine (n x cols, leading dimension n) and is empty here
  const double* dev_x = nullptr;
};

// One conditioning set's model: X = [1 | smooth_1 | ... ] with one penalty
// block per smooth.
struct Design {
  int n = 0, q = 0, m = 0;
  std::vector<int> S;                       // conditioning columns (sorted as given)
  std::vector<double> X;                    // n x q
  std::vector<std::vector<double>> blocks;  // dim_j x dim_j
  std::vector<int> offsets, dims, ranks;
  std::vector<double> initial_log_sp;       // m
  // geometry
  std::vector<double> Q;                    // n x q, X = Q R
  std::vector<double> R;                    // q x q upper triangular
  // single penalty (m == 1): whitened-penalty spectrum
  std::vector<double> spec;                 // q hat eigenvalues e_k (descending, >= 0)
  std::vector<double> QW;                   // n x q: Q * W, W the whitened eigenvectors
  // several penalties: per block root (dim_j x rank_j), root root' = S_j
  std::vector<std::vector<double>> roots;
  // additive designs of the design cache: X, Q and R are not formed on the
  // host; the device gathers X from these bases and factors it
  bool device_geometry = false;
  std::vector<std::shared_ptr<const Smooth>> parts;
};

// Thin-plate set-up in three parts, so that the top-k eigen problem of the
// eta matrix can be solved elsewhere (the device batches it per level):
// prepare (unique locations, polynomial null-space basis), the eta matrix,
// and finish (constraint absorption, scaling, centering) from its top-k
// eigenpairs (descending, largest-magnitude entry of each vector positive).
class DesignCache;

struct TprsPrep {
  int n = 0, d = 0, k = 0, m = 0, M = 0, nu = 0;
  std::vector<double> u;      // nu x d unique (shifted) locations, column-major
  std::vector<int> mapping;   // row -> unique location
  std::vector<double> T;      // nu x M polynomial null-space basis
};
TprsPrep tprs_prepare(const double* cols, int n, int d, int k);
std::vector<double> tprs_eta_matrix(const TprsPrep& prep);
double tprs_eta0(int d);  // eta constant of the default order for dimension d
Smooth tprs_finish(const TprsPrep& prep, const std::vector<double>& vals, const std::vector<double>& U);
Smooth build_smooth(const double* cols, int n, int d, int k);
double r_mean(const double* v, int n);
std::vector<double> initial_sp(const Design& des);
// initial.sp from the sums of squares of the columns of X (q)
std::vector<double> initial_sp_from_colsq(const Design& des, const std::vector<double>& xdiag);
// root (dim x rank) of a symmetric penalty block: root root' = block
std::vector<double> penalty_root(const std::vector<double>& block, int dim, int rank);
void prepare_geometry(Design* des);
// An additive (|S| >= 3) design without X, Q or R: blocks, roots and
// initial.sp from the cache's univariate smooths (device_geometry set).
std::shared_ptr<Design> build_additive_meta(int n, int p, const std::vector<int>& S, DesignCache* cache);
// A single-penalty (|S| <= 2) design without X, Q, QW or the spectrum: the
// smooth, its penalty and initial.sp (device_geometry set).
std::shared_ptr<Design> build_single_meta(int n, int p, const std::vector<int>& S, DesignCache* cache);
// sum of squares of each column of an n x cols matrix (long double accumulation)
std::vector<double> column_sumsq(const double* X, int n, int cols);

// Cache of univariate smooths (shared by every additive model containing the
// variable) and of full designs per conditioning set.
class DesignCache {
 public:
  DesignCache(const double* data, int n, int p) : data_(data), n_(n), p_(p) {}
  std::shared_ptr<const Design> get(const std::vector<int>& S);
  // Batched use from many threads: look every set up under one lock, build
  // the missing designs without the lock (build), insert them under one lock.
  std::vector<std::shared_ptr<const Design>> find_designs(const std::vector<const std::vector<int>*>& sets);
  std::shared_ptr<const Design> build(const std::vector<int>& S);
  void put_designs(const std::vector<const std::vector<int>*>& sets,
                   const std::vector<std::shared_ptr<const Design>>& designs);
  std::shared_ptr<const Smooth> univariate(int column);
  // bivariate thin-plate smooths built outside build_design (device eigen)
  void put_bivariate(const std::vector<int>& S, std::shared_ptr<const Smooth> smooth);
  // univariate smooths built outside the cache (device eigen)
  void put_univariate(int column, std::shared_ptr<const Smooth> smooth);
  bool has_univariate(int column);
  std::shared_ptr<const Smooth> bivariate(const std::vector<int>& S);
  bool has_design(const std::vector<int>& S);
  size_t size() const { return designs_.size(); }
  const double* data() const { return data_; }
  int n() const { return n_; }

 private:
  const double* data_;
  int n_, p_;
  std::mutex mu_;
  std::map<std::vector<int>, std::shared_ptr<const Design>> designs_;
  std::map<int, std::shared_ptr<const Smooth>> uni_;
  std::map<std::vector<int>, std::shared_ptr<const Smooth>> bi_;
};

std::shared_ptr<Design> build_design(const double* data, int n, int p, const std::vector<int>& S,
                                     DesignCache* cache);

}  // namespace fkpc
