"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset ships with the reference for these shapes, so inputs are
drawn from the nonlinear structural equation model the configurations name:
a random topological order; edge i -> j (i earlier) with probability
``edge_prob`` (optionally capped at ``max_in_degree`` parents); each node is
the sum over its parents of f(parent) with f drawn per edge from
{tanh(2u), sin(u), 0.5 u^2, u}, plus N(0, 0.5^2) noise; columns standardised
to mean 0, sd 1.
"""
import numpy as np

_FUNCS = (lambda u: np.tanh(2.0 * u), np.sin, lambda u: 0.5 * u * u, lambda u: u)


def nonlinear_sem(n, p, edge_prob, seed, max_in_degree=None):
    rs = np.random.default_rng(seed)
    order = rs.permutation(p)
    X = np.zeros((n, p))
    edges = []
    for pos, j in enumerate(order):
        parents = [int(i) for i in order[:pos] if rs.random() < edge_prob]
        if max_in_degree is not None and len(parents) > max_in_degree:
            parents = sorted(rs.choice(parents, size=max_in_degree, replace=False).tolist())
        v = rs.normal(0.0, 0.5, size=n)
        for i in parents:
            f = _FUNCS[int(rs.integers(len(_FUNCS)))]
            v = v + f(X[:, i])
        X[:, j] = v
        edges.extend((i, int(j)) for i in parents)
    X = (X - X.mean(axis=0)) / X.std(axis=0, ddof=1)
    return np.asfortranarray(X), edges


def ci_triples(p, count, seed, size_sampler):
    """``count`` random (x, y, S) triples; |S| from ``size_sampler(rs)``."""
    rs = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        k = int(size_sampler(rs))
        if k > p - 2:
            continue
        vars_ = rs.choice(p, size=k + 2, replace=False)
        x, y = int(vars_[0]), int(vars_[1])
        out.append((x, y, sorted(int(v) for v in vars_[2:])))
    return out


def level_batch_500x50(seed=2, count=4096):
    """n=500, p=50 nonlinear SEM (edge prob 0.08); ``count`` triples with |S|
    uniform on 0..4 -- the single-level CI batch microbenchmark."""
    X, _ = nonlinear_sem(500, 50, 0.08, seed)
    return X, ci_triples(50, count, seed + 1, lambda rs: rs.integers(0, 5))


def skeleton_200x10(seed=1):
    """n=200, p=10, edge prob 0.25: the CPU-runnable skeleton case."""
    return nonlinear_sem(200, 10, 0.25, seed)[0]


def skeleton_351x48(seed=3):
    """n=351, p=48, edge prob 0.1, at most 8 parents: the full-skeleton case."""
    return nonlinear_sem(351, 48, 0.1, seed, max_in_degree=8)[0]


def deep_skeleton_seed(levels_of, min_level=8, first=1, last=1000):
    """The first seed in [first, last] whose n=351, p=48 SEM (edge prob 0.1,
    at most 8 parents) gives a default-Inf skeleton that runs level
    ``min_level`` (a conditioning set of that size is tested), else the
    seed whose skeleton runs the most levels (the first of equals).
    ``levels_of(X)`` returns one plus the deepest level at which a skeleton
    on X ran a test.  Returns (seed, levels).  Over seeds 1..800 no skeleton
    reaches level 8 (the deepest run level 7: seeds 537 and 795), so the rule
    gives 537."""
    best = (None, -1)
    for seed in range(first, last + 1):
        levels = int(levels_of(skeleton_351x48(seed)))
        if levels - 1 >= min_level:
            return seed, levels
        if levels > best[1]:
            best = (seed, levels)
    return best


def uneven_batch_500x64(seed=4, count=16384):
    """n=500, p=64; |S| ~ geometric(0.35) truncated at 12 (permutation batch)."""
    X, _ = nonlinear_sem(500, 64, 0.08, seed)

    def size(rs):
        while True:
            k = int(rs.geometric(0.35)) - 1
            if k <= 12:
                return k
    return X, ci_triples(64, count, seed + 1, size)


def adjoint_targets_1000(seed=5, count=2048):
    """GCV adjoint / Newton selection workload: n=1000, p=50 SEM (edge prob
    0.08) and ``count`` (target, S) fits with |S| uniform on 3..8 (additive
    smooths, 3..8 log smoothing parameters, q = 1 + 9|S| up to 73)."""
    X, _ = nonlinear_sem(1000, 50, 0.08, seed)
    rs = np.random.default_rng(seed + 1)
    fits = []
    for _ in range(count):
        k = int(rs.integers(3, 9))
        cols = rs.choice(50, size=k + 1, replace=False)
        fits.append((int(cols[0]), sorted(int(c) for c in cols[1:])))
    return X, fits


# Seeds of the n=351, p=48 full-skeleton rows: the deepest-skeleton seed
# (deep_skeleton_seed) and seed 3.
SKELETON_351X48_SEEDS = (537, 3)


def orientation_collider_free(n=300, p=12, edge_prob=0.25, seed=2, max_in_degree=4):
    """An orientation input with no colliders: the SEM's true skeleton, and
    for every non-adjacent pair a separating set of all other nodes (so no
    v-structure is oriented and every undirected neighbourhood goes through
    the regrVonPS stage).  Returns (X, adjacency p x p bool, sepsets
    {(a, b): S})."""
    X, edges = nonlinear_sem(n, p, edge_prob, seed, max_in_degree=max_in_degree)
    adj = np.zeros((p, p), dtype=bool)
    for i, j in edges:
        adj[i, j] = adj[j, i] = True
    sepsets = {(a, b): [c for c in range(p) if c not in (a, b)]
               for a in range(p) for b in range(p) if a != b and not adj[a, b]}
    return X, adj, sepsets


ORIENTATION_CASES = {
    # name: (generator, kwargs)
    "free300x12_s2": dict(n=300, p=12, edge_prob=0.25, seed=2),
    "free351x24_s4": dict(n=351, p=24, edge_prob=0.2, seed=4),
}
