"""R-compatible random streams for the permutation CI methods (oracle).

TEST INFRASTRUCTURE ONLY: this module is the CPU checker for the library's
permutation streams.  Nothing in the shipped library imports it.

What it restates (published algorithms, written from their descriptions):

* MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998) with R's
  ``set.seed`` seeding: 50 rounds of the LCG ``seed = 69069*seed + 1`` to
  scramble the user seed, then 625 further LCG values fill the state
  (element 0 is the position counter, set to 624) -- R's documented
  ``RNGkind("Mersenne-Twister")`` behaviour.
* ``unif_rand``: the tempered 32-bit output times 2^-32, nudged into (0,1).
* ``R_unif_index`` with ``sample.kind = "Rejection"``: draw 16-bit chunks
  ``floor(u * 65536)`` until the masked value is below the bound.
* ``norm_rand`` by inversion (R's default ``normal.kind``), used only to pin
  the stream against the reference's 500x50 fixture data.

Reference call sites: fastkpc/src/full_cuda_ci_one_call.cpp:464-567 (the
permutation table builder for dcc.perm / hsic.perm) and
kpcalg/R/hsicperm.R:82 (``sample(n)``).
"""
import math

import numpy as np

_N = 624
_M = 397
_MATRIX_A = 0x9908B0DF
_UPPER = 0x80000000
_LOWER = 0x7FFFFFFF
_I2_32M1 = 2.328306437080797e-10


class RStream:
    """R's Mersenne-Twister stream after ``set.seed(seed)``."""

    def __init__(self, seed):
        s = seed & 0xFFFFFFFF
        for _ in range(50):
            s = (69069 * s + 1) & 0xFFFFFFFF
        state = []
        for _ in range(_N + 1):
            s = (69069 * s + 1) & 0xFFFFFFFF
            state.append(s)
        self.mt = state[1:]
        self.mti = _N
        self.draws = 0

    def _refill(self):
        mt = self.mt
        for kk in range(_N):
            y = (mt[kk] & _UPPER) | (mt[(kk + 1) % _N] & _LOWER)
            v = mt[(kk + _M) % _N] ^ (y >> 1)
            if y & 1:
                v ^= _MATRIX_A
            mt[kk] = v
        self.mti = 0

    def genrand(self):
        if self.mti >= _N:
            self._refill()
        y = self.mt[self.mti]
        self.mti += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return (y & 0xFFFFFFFF) * 2.3283064365386963e-10

    def unif_rand(self):
        self.draws += 1
        x = self.genrand()
        if x <= 0.0:
            return 0.5 * _I2_32M1
        if 1.0 - x <= 0.0:
            return 1.0 - 0.5 * _I2_32M1
        return x

    def unif_index(self, dn):
        """R_unif_index(dn) under sample.kind = "Rejection"."""
        if dn <= 0:
            return 0
        bits = int(math.ceil(math.log2(dn)))
        while True:
            v = 0
            for _ in range(0, bits + 1, 16):
                v = 65536 * v + int(math.floor(self.unif_rand() * 65536.0))
            v &= (1 << bits) - 1
            if v < dn:
                return v

    def norm_rand(self):
        """Inversion: R's default normal generator (BIG = 2^27)."""
        from scipy.special import ndtri
        big = 134217728.0
        u = self.unif_rand()
        u = int(big * u) + self.unif_rand()
        return float(ndtri(u / big))


def dcc_permutations(stream, n, replicates):
    """energy::dcov.test permutations: one vector mutated across replicates.

    Each replicate does n-1 swaps: pick j = floor(u * remaining), then swap
    positions j and remaining-1 (fastkpc/src/full_cuda_ci_one_call.cpp:500-521).
    Returns an int32 array (replicates, n).
    """
    perm = list(range(n))
    out = np.empty((replicates, n), dtype=np.int32)
    for r in range(replicates):
        remaining = n
        for _ in range(n - 1):
            j = int(math.floor(stream.unif_rand() * remaining))
            j = min(max(j, 0), remaining - 1)
            remaining -= 1
            perm[j], perm[remaining] = perm[remaining], perm[j]
        out[r] = perm
    return out


def hsic_permutations(stream, n, replicates):
    """``sample(n)`` per replicate (R_unif_index on a shrinking pool).

    Output position i takes pool[j], then pool[j] = pool[last]
    (fastkpc/src/full_cuda_ci_one_call.cpp:524-560).  Returns (replicates, n).
    """
    out = np.empty((replicates, n), dtype=np.int32)
    for r in range(replicates):
        pool = list(range(n))
        remaining = n
        for i in range(n):
            j = stream.unif_index(remaining)
            out[r, i] = pool[j]
            remaining -= 1
            pool[j] = pool[remaining]
    return out
