// R-compatible uniform stream for the permutation CI methods.
//
// MT19937 (Matsumoto & Nishimura 1998) seeded the way R's set.seed() does for
// RNGkind("Mersenne-Twister"): the seed is scrambled by 50 rounds of
// seed = 69069 seed + 1, then 625 further values fill the state, whose first
// word (the position) is reset to 624.  unif_rand() is the tempered output
// times 2^-32 kept inside (0, 1); R_unif_index() under sample.kind =
// "Rejection" draws 16-bit chunks floor(u * 65536) until the masked value is
// below the bound.  Permutation tables follow the reference's builder
// (fastkpc/src/full_cuda_ci_one_call.cpp:464-567): dcc.perm mutates one
// vector with n-1 swaps per replicate (energy's dCOVtest), hsic.perm draws
// sample(n) from a shrinking pool.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace fkpc {

class RStream {
 public:
  explicit RStream(uint32_t seed) {
    uint32_t s = seed;
    for (int j = 0; j < 50; ++j) s = 69069u * s + 1u;
    for (int j = 0; j < 625; ++j) {
      s = 69069u * s + 1u;
      if (j > 0) mt_[j - 1] = s;
    }
    mti_ = 624;
  }

  double unif_rand() {
    ++draws_;
    const double x = genrand();
    const double i2_32m1 = 2.328306437080797e-10;
    if (x <= 0.0) return 0.5 * i2_32m1;
    if (1.0 - x <= 0.0) return 1.0 - 0.5 * i2_32m1;
    return x;
  }

  int unif_index(int dn) {
    if (dn <= 0) return 0;
    // ceil(log2(dn)) as R computes it in double, exact for every int dn >= 1:
    // the bit length of dn - 1
    const int bits = dn == 1 ? 0 : 32 - __builtin_clz(static_cast<unsigned>(dn - 1));
    for (;;) {
      int64_t v = 0;
      for (int k = 0; k <= bits; k += 16) v = 65536 * v + static_cast<int64_t>(std::floor(unif_rand() * 65536.0));
      v &= (static_cast<int64_t>(1) << bits) - 1;
      if (v < dn) return static_cast<int>(v);
    }
  }

  // replicates x n table for one dcc.perm test
  void dcc_permutations(int n, int replicates, int* out) {
    dcc_swaps(n, replicates, out);
    dcc_assemble(n, replicates, out, &perm_);
  }

  // replicates x n table for one hsic.perm test
  void hsic_permutations(int n, int replicates, int* out) {
    hsic_draws(n, replicates, out);
    hsic_assemble(n, replicates, out, &pool_);
  }

  // The two tables in two passes: the stream's part (the draws, in stream
  // order, into the table's rows) and the part that uses no stream (turning
  // a row's draws into its permutation), which may run for many tests at
  // once.  dcc.perm: swap k of a replicate takes j = floor(u (n - k)) and
  // exchanges entries j and n - 1 - k of one vector carried from replicate
  // to replicate; hsic.perm: draw i takes R_unif_index(n - i) from a pool
  // that each replicate starts afresh.
  void dcc_swaps(int n, int replicates, int* out) {
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      int remaining = n;
      for (int k = 0; k < n - 1; ++k) {
        int j = static_cast<int>(std::floor(unif_rand() * remaining));
        if (j < 0) j = 0;
        if (j >= remaining) j = remaining - 1;
        --remaining;
        row[k] = j;
      }
    }
  }
  static void dcc_assemble(int n, int replicates, int* out, std::vector<int>* scratch) {
    std::vector<int>& perm = *scratch;
    perm.resize(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      int remaining = n;
      for (int k = 0; k < n - 1; ++k) {
        const int j = row[k];
        --remaining;
        const int t = perm[j];
        perm[j] = perm[remaining];
        perm[remaining] = t;
      }
      for (int i = 0; i < n; ++i) row[i] = perm[i];
    }
  }
  void hsic_draws(int n, int replicates, int* out) {
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      for (int i = 0; i < n; ++i) row[i] = unif_index(n - i);
    }
  }
  static void hsic_assemble(int n, int replicates, int* out, std::vector<int>* scratch) {
    std::vector<int>& pool = *scratch;
    pool.resize(n);
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      for (int i = 0; i < n; ++i) pool[i] = i;
      int remaining = n;
      for (int i = 0; i < n; ++i) {
        const int j = row[i];
        row[i] = pool[j];
        --remaining;
        pool[j] = pool[remaining];
      }
    }
  }

  uint64_t draws() const { return draws_; }

 private:
  double genrand() {
    static const uint32_t mag01[2] = {0u, 0x9908b0dfu};
    if (mti_ >= 624) {
      int kk = 0;
      for (; kk < 624 - 397; ++kk) {
        const uint32_t y = (mt_[kk] & 0x80000000u) | (mt_[kk + 1] & 0x7fffffffu);
        mt_[kk] = mt_[kk + 397] ^ (y >> 1) ^ mag01[y & 1u];
      }
      for (; kk < 623; ++kk) {
        const uint32_t y = (mt_[kk] & 0x80000000u) | (mt_[kk + 1] & 0x7fffffffu);
        mt_[kk] = mt_[kk + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1u];
      }
      const uint32_t y = (mt_[623] & 0x80000000u) | (mt_[0] & 0x7fffffffu);
      mt_[623] = mt_[396] ^ (y >> 1) ^ mag01[y & 1u];
      mti_ = 0;
    }
    uint32_t y = mt_[mti_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return static_cast<double>(y) * 2.3283064365386963e-10;
  }

  uint32_t mt_[624];
  int mti_;
  uint64_t draws_ = 0;
  std::vector<int> perm_, pool_;
};

}  // namespace fkpc
