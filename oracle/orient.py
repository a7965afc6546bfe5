"""WAN-PDAG orientation of a kernel-PC skeleton (oracle).

TEST INFRASTRUCTURE ONLY: the CPU checker for the library's orientation
(``fkpc_orient_wanpdag``).  A restatement of kpcalg's ``udag2wanpdag``
(kpcalg/R/udag2wanpdag.R:104-437) with the defaults the reference's strict
pipeline runs it with -- ``fast_kpc()`` orients through
``fastkpc_orient_wanpdag_kpcalg_authority`` (fastkpc/R/fast_kpc.R:263-330,
:499-511): the skeleton's alpha, numCol and CI method, no unfaithful-triple
list, solve.confl = FALSE, all three rules -- and of ``regrVonPS``
(kpcalg/R/regrvonps.R:17-39).

pdag[i, j] = 1 and pdag[j, i] = 0 is the edge i -> j; both 1 is undirected.
Indices are 0-based.  The iteration orders are R's: ``which(M, arr.ind =
TRUE)`` walks a matrix column by column, ``combn`` gives combinations in
lexicographic order of positions.

* Colliders (:296-324): for each (x, y) with g[x, y] = 1 in column-major
  order and each other neighbour z of y (ascending), x, z non-adjacent and y
  in neither sepset(x, z) nor sepset(z, x): x -> y <- z.
* Neighbourhoods (:326-429): for s = 1, 2, ... while some node has s or more
  undirected neighbours, for each node V whose undirected neighbourhood has
  exactly s members (or fewer, once V was updated), for s2 from that size
  down to 1 and each s2-subset S of it (``checkImmor`` first): regress V on
  S and its parents; if the residual is dependent on some member of S
  (``regrVonPS`` counts p < alpha) the orientation S -> V is rejected;
  otherwise it is also rejected when some W in S, with a subset S2 of its
  own undirected neighbourhood containing V, can be regressed to
  independence of S2; an accepted orientation sets S -> V and V -> the rest
  of V's undirected neighbours, then rules 1-3 run to a fixed point.
  As in R, the subsets of V's neighbourhood listed before an accepted
  orientation are still tried after it (the reference's native C++ engine,
  fastkpc/src/wanpdag_engine.cpp:369-390, stops at the first accepted one);
  the reverse tests stop at the first W that decides (R runs the rest, whose
  outcome cannot change the decision).
* ``regrVonPS``: residual of data[:, V] on data[:, S + parents(V)] by the
  kernel-PC regression (``regrXonS``), then the CI test of that residual
  against each data[:, s], s in S, with no conditioning set.

Parity pin: ``oracle.gcv`` and ``oracle.skeleton`` are pinned by their own
fixtures; the graph logic here has no reference output to pin it (kpcalg's R
and its packages are absent), so its rules are also checked on hand-built
graphs in the CPU tests.
"""
import itertools

import numpy as np

from . import skeleton as skel_mod
from . import gcv, tprs


def _which_cm(mask):
    """(row, col) pairs of a boolean matrix in R's column-major order."""
    p = mask.shape[0]
    return [(i, j) for j in range(p) for i in range(p) if mask[i, j]]


def _combn(values, k):
    """R's combn(values, k) columns; a single value gives itself."""
    values = list(values)
    if len(values) == 1:
        return [values]
    return [list(c) for c in itertools.combinations(values, k)]


def _undirected_nbhd(pdag):
    p = pdag.shape[0]
    und = (pdag == 1) & (pdag.T == 1)
    return [[j for j in range(p) if und[i, j]] for i in range(p)]


def _parents(pdag, v):
    return [i for i in range(pdag.shape[0]) if pdag[i, v] == 1 and pdag[v, i] == 0]


def check_immor(pdag, v, S):
    """kpcalg's checkImmor (udag2wanpdag.R:278-293)."""
    udag = np.minimum(pdag + pdag.T, 1)
    par = _parents(pdag, v)
    if len(S) > 1:
        t1 = udag[np.ix_(S, S)] + np.eye(len(S), dtype=udag.dtype)
        if np.any((t1 == 0) & (t1.T == 0)):
            return False
    if par and np.sum(udag[np.ix_(par, S)]) < len(S) * len(par):
        return False
    return True


def _set(pdag, a, b):
    """a -> b; True when the matrix changed."""
    changed = pdag[a, b] != 1 or pdag[b, a] != 0
    pdag[a, b] = 1
    pdag[b, a] = 0
    return bool(changed)


def rule1(pdag):
    """Rule 1 (udag2wanpdag.R:115-168): a -> b - c, a and c non-adjacent: b -> c.
    Returns the number of edges it changed."""
    count = 0
    for a, b in _which_cm((pdag == 1) & (pdag.T == 0)):
        isC = [c for c in range(pdag.shape[0])
               if pdag[b, c] == 1 and pdag[c, b] == 1 and pdag[a, c] == 0 and pdag[c, a] == 0]
        for c in isC:
            count += _set(pdag, b, c)
    return count


def rule2(pdag):
    """Rule 2 (:169-193): a - b with a chain a -> c -> b: a -> b."""
    count = 0
    for a, b in _which_cm((pdag == 1) & (pdag.T == 1)):
        isC = [c for c in range(pdag.shape[0])
               if pdag[a, c] == 1 and pdag[c, a] == 0 and pdag[c, b] == 1 and pdag[b, c] == 0]
        for _ in isC:
            count += _set(pdag, a, b)
    return count


def rule3(pdag):
    """Rule 3 (:195-261): a - b, a - c1 -> b, a - c2 -> b, c1 and c2
    non-adjacent: a -> b."""
    count = 0
    for a, b in _which_cm((pdag == 1) & (pdag.T == 1)):
        cs = [c for c in range(pdag.shape[0])
              if pdag[a, c] == 1 and pdag[c, a] == 1 and pdag[c, b] == 1 and pdag[b, c] == 0]
        if len(cs) >= 2:
            for c1, c2 in itertools.combinations(cs, 2):
                if pdag[c1, c2] == 0 and pdag[c2, c1] == 0:
                    count += _set(pdag, a, b)
                    break
    return count


def regr_v_on_ps(data, pdag, v, S, method, alpha, num_col=35, sig=1.0, trace=None, context=0, cache=None):
    """kpcalg's regrVonPS (regrvonps.R:17-39): the number of members s of S
    whose test of (residual of v on S + parents(v), data[:, s]) has p < alpha.
    The conditioning set is sorted (the reference's native form sorts it too,
    fastkpc/src/regrvonps_native.cpp:40-69; the fit does not depend on the
    order of its covariates).  ``cache`` maps (v, Z) to the residual."""
    Z = tuple(sorted(list(S) + _parents(pdag, v)))
    r = None if cache is None else cache.get((v, Z))
    if r is None:
        prep = gcv.Prepared(tprs.design(data, list(Z)))
        r, _ = gcv.fit(prep, data[:, v])
        if cache is not None:
            cache[(v, Z)] = r
    rc = skel_mod.ResidualCache(np.column_stack([r] + [data[:, s] for s in S]))
    count = 0
    for k in range(len(S)):
        pv = skel_mod.ci_pvalue(rc, method, 0, k + 1, [], num_col, sig)
        if trace is not None:
            trace.append({"reverse": context, "target": v, "other": S[k], "S": list(S), "Z": list(Z),
                          "p": pv, "rejected": pv < alpha})
        if pv < alpha:
            count += 1
    return count


def orient(data, adjacency, sepsets, method="dcc.gamma", alpha=0.1, num_col=35, sig=1.0, regress=None):
    """The WAN-PDAG of a skeleton: adjacency (p x p bool), sepsets {(x, z): S}.
    ``regress(pdag, v, S, context)`` may replace ``regr_v_on_ps`` (same
    contract; context 0 for V's own test, 1 for the reverse test of a W).
    Returns (pdag int matrix, trace of the regrVonPS tests, counts)."""
    g = np.asarray(adjacency, dtype=np.int64)
    p = g.shape[0]
    pdag = g.copy()
    trace = []
    counts = {"collider": 0, "rule1": 0, "rule2": 0, "rule3": 0, "generalized": 0, "regrvonps_calls": 0}
    cache = {}
    if regress is None:
        def regress(pd, v, S, context):
            return regr_v_on_ps(data, pd, v, S, method, alpha, num_col, sig, trace, context, cache)

    def call(pd, v, S, context):
        counts["regrvonps_calls"] += 1
        return regress(pd, v, S, context)

    if g.sum() == 0:
        return pdag, trace, counts
    for x, y in _which_cm(g == 1):
        for z in [z for z in range(p) if g[y, z] == 1 and z != x]:
            sep = list(sepsets.get((x, z), [])) + list(sepsets.get((z, x), []))
            if g[x, z] == 0 and y not in sep:
                changed = _set(pdag, x, y)
                changed = _set(pdag, z, y) or changed
                counts["collider"] += int(changed)
    s = 1
    nbhd = _undirected_nbhd(pdag)
    size = [len(v) for v in nbhd]
    updated = [False] * p
    while max(size) >= s:
        for V in range(p):
            s2 = s
            if size[V] == s2 or (size[V] < s2 and updated[V]):
                s2 = size[V]
                while s2 > 0:
                    # the subsets of the neighbourhood as it was when this size began;
                    # after an accepted orientation the remaining ones are still tried
                    for S in _combn(nbhd[V], s2):
                        to_update = True
                        if not check_immor(pdag, V, S):
                            continue
                        if call(pdag, V, S, 0) > 0:
                            to_update = False
                        else:
                            for W in S:
                                s3 = size[W]
                                go_on = True
                                while go_on and s3 > 0:
                                    for S2 in _combn(nbhd[W], s3):
                                        if not to_update:
                                            break  # later tests cannot change the outcome
                                        if check_immor(pdag, W, S2) and S2.count(V) == 1:
                                            if call(pdag, W, S2, 1) == 0:
                                                to_update = False
                                                go_on = False
                                    s3 -= 1
                                if not to_update:
                                    break
                        if to_update:
                            counts["generalized"] += 1
                            pdag[V, S] = 0
                            pdag[S, V] = 1
                            rest = [u for u in nbhd[V] if u not in S]
                            if rest:
                                pdag[rest, V] = 0
                                pdag[V, rest] = 1
                            s2 = 0
                            while True:
                                old = pdag.copy()
                                counts["rule1"] += rule1(pdag)
                                counts["rule2"] += rule2(pdag)
                                counts["rule3"] += rule3(pdag)
                                if np.array_equal(pdag, old):
                                    break
                            nbhd = _undirected_nbhd(pdag)
                            updated[V] = True
                            size = [len(v) for v in nbhd]
                    s2 -= 1
        s += 1
    return pdag, trace, counts
