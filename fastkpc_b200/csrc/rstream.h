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

  // R_unif_index(dn) under sample.kind "Rejection".  unif_rand() is y 2^-32
  // for the tempered word y (y = 0 lifted to 2^-33), so floor(u 65536), R's
  // 16-bit chunk, is exactly y >> 16: the chunks come straight from the words.
  int unif_index(int dn) {
    if (dn <= 0) return 0;
    // ceil(log2(dn)) as R computes it in double, exact for every int dn >= 1:
    // the bit length of dn - 1
    const int bits = dn == 1 ? 0 : 32 - __builtin_clz(static_cast<unsigned>(dn - 1));
    const int64_t mask = (static_cast<int64_t>(1) << bits) - 1;
    for (;;) {
      int64_t v = 0;
      for (int k = 0; k <= bits; k += 16) {
        ++draws_;
        v = 65536 * v + static_cast<int64_t>(genword() >> 16);
      }
      v &= mask;
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
  // floor(u m) for u = y 2^-32 is (y m) >> 32 while y m stays below 2^53
  // (m < 2^21): the product and its scaling are exact in double (y = 0, lifted
  // to 2^-33, gives 0 either way).
  void dcc_swaps(int n, int replicates, int* out) {
    const bool exact = n < (1 << 21);
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      int remaining = n;
      for (int k = 0; k < n - 1; ++k) {
        int j;
        if (exact) {
          ++draws_;
          j = static_cast<int>((static_cast<uint64_t>(genword()) * static_cast<uint64_t>(remaining)) >> 32);
        } else {
          j = static_cast<int>(std::floor(unif_rand() * remaining));
          if (j < 0) j = 0;
          if (j >= remaining) j = remaining - 1;
        }
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
  // hsic.perm's draws word by word, without a branch on the rejection: every
  // word is written to the current slot and the slot advances when the word
  // is accepted (R_unif_index(dn) takes one word per attempt while dn <= 2^15).
  void hsic_draws(int n, int replicates, int* out) {
    for (int r = 0; r < replicates; ++r) {
      int* row = out + static_cast<int64_t>(r) * n;
      if (n > (1 << 15)) {
        for (int i = 0; i < n; ++i) row[i] = unif_index(n - i);
        continue;
      }
      int i = 0;
      while (i < n) {
        const int dn = n - i;
        const uint32_t mask = dn == 1 ? 0u : (0xffffffffu >> __builtin_clz(static_cast<unsigned>(dn - 1)));
        const int v = static_cast<int>((genword() >> 16) & mask);
        ++draws_;
        row[i] = v;
        i += v < dn ? 1 : 0;
      }
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
  double genrand() { return static_cast<double>(genword()) * 2.3283064365386963e-10; }

  // the next tempered MT19937 word
  uint32_t genword() {
    if (mti_ >= 624) refill();
    return tw_[mti_++];
  }

  // The next 624 words: the state's twist (the tap 0x9908b0df applied by a
  // mask, without a table), then all 624 tempered at once into tw_.
  void refill() {
    auto twist = [](uint32_t hi, uint32_t lo, uint32_t far) {
      const uint32_t y = (hi & 0x80000000u) | (lo & 0x7fffffffu);
      return far ^ (y >> 1) ^ (0x9908b0dfu & (0u - (y & 1u)));
    };
    int kk = 0;
    for (; kk < 624 - 397; ++kk) mt_[kk] = twist(mt_[kk], mt_[kk + 1], mt_[kk + 397]);
    for (; kk < 623; ++kk) mt_[kk] = twist(mt_[kk], mt_[kk + 1], mt_[kk + (397 - 624)]);
    mt_[623] = twist(mt_[623], mt_[0], mt_[396]);
    for (int i = 0; i < 624; ++i) {
      uint32_t y = mt_[i];
      y ^= y >> 11;
      y ^= (y << 7) & 0x9d2c5680u;
      y ^= (y << 15) & 0xefc60000u;
      y ^= y >> 18;
      tw_[i] = y;
    }
    mti_ = 0;
  }

  uint32_t mt_[624];
  uint32_t tw_[624];  // the current block of tempered words
  int mti_;
  uint64_t draws_ = 0;
  std::vector<int> perm_, pool_;
};

}  // namespace fkpc
