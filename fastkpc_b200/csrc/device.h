// Device-side descriptors shared by the host runtime and the kernels.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define FKPC_HD __host__ __device__
#else
#define FKPC_HD
#endif

namespace fkpc {

constexpr int kMaxPenalties = 62;     // |S| <= 62 (p <= 64), design widths up to q = 559
constexpr int kCtaPenalties = 12;     // the shared-memory CTA fit classes: |S| <= 12
constexpr int kWideQ = 560;           // the wide fit class: q <= 560 coefficients,
constexpr int kWideR = 496;           // at most 496 stacked penalty-root rows
constexpr int kMaxSingleQ = 32;       // single-penalty designs have q in {10, 30}
constexpr int kStatusOk = 0;
constexpr int kStatusNumeric = 3;
constexpr int kStatusNotConverged = 4;
constexpr int kStatusRank = 5;
constexpr int kStatusInvalid = 1;
constexpr unsigned int FKPC_FLAG_GUARDED_DEV = 1u;  // matches FKPC_FLAG_GUARDED
constexpr unsigned int FKPC_FLAG_DIRECT_DEV = 2u;   // matches FKPC_FLAG_DIRECT
constexpr int kFitFlagRankTruncated = 1;            // FitResult.flags: the rank rule dropped a coefficient

// Warp-per-fit class of additive designs: q <= kWarpQ coefficients, at most
// kWarpR stacked penalty rows and kWarpM penalties.
constexpr int kWarpQ = 40;
constexpr int kWarpR = 32;
constexpr int kWarpM = 4;
constexpr int kWarpTri = kWarpQ * (kWarpQ + 1) / 2;

// Row-packed upper triangle of width kWarpQ: row t holds columns t..kWarpQ-1.
FKPC_HD constexpr int packed_row(int t, int c) { return t * (2 * kWarpQ - t + 1) / 2 + (c - t); }

// One conditioning set's geometry, resident in a device arena of doubles,
// for at most MP penalties.
template <int MP>
struct DesignT {
  int kind;        // 1: single penalty (spectral), 2: several penalties (augmented QR)
  int q;           // coefficients
  int m;           // penalties
  int rsum;        // sum of penalty ranks (rows of the stacked penalty root)
  int64_t basis;   // kind 1: QW (n x q); kind 2: Q (n x q)
  int64_t rmat;    // kind 2: R (q x q column-major, upper triangular)
  int64_t spec;    // kind 1: hat eigenvalues e (q)
  int64_t roots;   // kind 2: penalty roots, block j dim_j x rank_j column-major, consecutive
  int64_t rpack;   // kind 2 with q <= kWarpQ: R row-packed (kWarpTri doubles, zero beyond q), else -1
  int64_t ext;     // m > kCtaPenalties: arena offset of the design's WideDesign (all m blocks), else -1
  int off[MP];
  int dim[MP];
  int rank[MP];
  int rowoff[MP];    // first stacked-root row of block j
  int rootoff[MP];   // offset of block j's root inside ``roots``
  double log_sp0[MP];
};
// The descriptor array every kernel indexes: the blocks of designs with
// m <= kCtaPenalties; a wider design keeps its header here and its full
// descriptor (a WideDesign) in the arena at ``ext``.
using DesignDev = DesignT<kCtaPenalties>;
using WideDesign = DesignT<kMaxPenalties>;
// The warp fit class's copy in shared memory (m <= kWarpM).
using WarpDesign = DesignT<kWarpM>;
static_assert(sizeof(WideDesign) % sizeof(double) == 0, "wide descriptors are copied into the arena as doubles");

// One additive design whose geometry the device builds: X = [1 | B_1 | ...]
// gathered from the univariate smooth bases, X = Q R by Householder, Q and R
// (and row-packed R) written to the arena.
template <int MP>
struct GeomJobT {
  int64_t basis;                 // arena offset of Q (n x q)
  int64_t rmat;                  // arena offset of R (q x q)
  int64_t rpack;                 // arena offset of row-packed R, or -1
  const double* src[MP];         // smooth j's basis (n x dim_j, leading dimension n), device memory
  int off[MP];
  int dim[MP];
  int q;
  int m;
};
using GeomJob = GeomJobT<kCtaPenalties>;
using WideGeomJob = GeomJobT<kMaxPenalties>;

// One single-penalty design whose geometry the device builds: X = [1 | B],
// B the smooth's basis, S its penalty; QW and the spectrum to the arena.
struct SingleGeomJob {
  int64_t basis;   // arena offset of QW (n x q)
  int64_t spec;    // arena offset of the spectrum (q)
  const double* src;  // B (n x (q - 1), leading dimension n), device memory
  const double* pen;  // S ((q - 1) x (q - 1)), device memory
  int q;
  int rank;
};

// One residual fit: data column ``column`` regressed on design ``design``.
struct FitJob {
  int design;
  int column;
  int out;         // residual slot (column of the residual slab)
  int pad;
};

struct FitResult {
  double log_sp[kCtaPenalties];  // the first kCtaPenalties (a wide fit writes all m to a buffer of its own)
  double score;
  double edf;
  double rss;
  int status;
  int iterations;
  int evaluations;
  int flags;
};

// Optimiser state of a warp-class fit handed from fit_multi_warp_kernel to
// the speculative continuation kernel at the start of a Newton iteration.
struct FitState {
  double log_sp[kWarpM];
  double newton[kWarpM];
  double steep[kWarpM];
  double gradient[kWarpM];
  double hess[kWarpM * kWarpM];
  double min_score;
  double score_red;
  int it;
  int calls;
  int steepest;
  int pad;
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
