// Device-side descriptors shared by the host runtime and the kernels.
#pragma once
#include <cstdint>

namespace fkpc {

constexpr int kMaxPenalties = 8;      // |S| <= 8 in the shared-memory multi-penalty kernel
constexpr int kMaxSingleQ = 32;       // single-penalty designs have q in {10, 30}
constexpr int kStatusOk = 0;
constexpr int kStatusNumeric = 3;
constexpr int kStatusNotConverged = 4;
constexpr int kStatusRank = 5;
constexpr int kStatusInvalid = 1;
constexpr unsigned int FKPC_FLAG_GUARDED_DEV = 1u;  // matches FKPC_FLAG_GUARDED
constexpr unsigned int FKPC_FLAG_DIRECT_DEV = 2u;   // matches FKPC_FLAG_DIRECT

// One conditioning set's geometry, resident in a device arena of doubles.
struct DesignDev {
  int kind;        // 1: single penalty (spectral), 2: several penalties (augmented QR)
  int q;           // coefficients
  int m;           // penalties
  int rsum;        // sum of penalty ranks (rows of the stacked penalty root)
  int64_t basis;   // kind 1: QW (n x q); kind 2: Q (n x q)
  int64_t rmat;    // kind 2: R (q x q column-major, upper triangular)
  int64_t spec;    // kind 1: hat eigenvalues e (q)
  int64_t roots;   // kind 2: penalty roots, block j dim_j x rank_j column-major, consecutive
  int off[kMaxPenalties];
  int dim[kMaxPenalties];
  int rank[kMaxPenalties];
  int rowoff[kMaxPenalties];    // first stacked-root row of block j
  int rootoff[kMaxPenalties];   // offset of block j's root inside ``roots``
  double log_sp0[kMaxPenalties];
};

// One residual fit: data column ``column`` regressed on design ``design``.
struct FitJob {
  int design;
  int column;
  int out;         // residual slot (column of the residual slab)
  int pad;
};

struct FitResult {
  double log_sp[kMaxPenalties];
  double score;
  double edf;
  double rss;
  int status;
  int iterations;
  int evaluations;
  int flags;
};

// One CI test: statistic between two residual components.
struct PairJob {
  int left;        // component index
  int right;
  int out;         // record index
  int pad;
};

struct RecordDev {
  double p_value;
  double p_exact;
  double statistic;
  double mean;
  double variance;
  int status;
  unsigned int flags;
};

}  // namespace fkpc
