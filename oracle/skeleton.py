"""pcalg-stable skeleton replay over the CI oracle (oracle).

TEST INFRASTRUCTURE ONLY: the CPU checker for the library's skeleton runner.

* level plan (fastkpc/src/skeleton_task_scheduler.cpp:70-132): for every
  edge x<y of the level-start adjacency, the x-side tasks (S over
  combinations of adj(x)\\{y} of size ``level``) then the y-side tasks; the
  first task of a side "opens the next level" when that side has more than
  ``level`` neighbours.
* replay (fastkpc/src/full_cuda_ci_one_call.cpp:5229-5579): per edge, tasks
  run in plan order until one deletes (p >= alpha); the trailing tasks of that
  edge are skipped.  pMax keeps the max p per edge, sepsets record the
  deleting S, deletions apply at level end; the run stops when no executed
  task opens the next level or the level exceeds m.max.
* permutation methods consume one global R stream in pcalg order: ordered by
  (x, y, S lexicographic) over the executed tasks
  (fastkpc/src/full_cuda_ci_one_call.cpp:327-337, :5301-5335).
"""
import itertools

import numpy as np

from . import gcv, rng, stats, tprs


def make_layer_plan(adj, level):
    p = adj.shape[0]
    tasks = []
    for x in range(p - 1):
        for y in range(x + 1, p):
            if not adj[x, y]:
                continue
            for (a, b) in ((x, y), (y, x)):
                nb = [i for i in range(p) if i != b and adj[i, a]]
                first = True
                for S in itertools.combinations(nb, level):
                    tasks.append({"edge": (x, y), "x": a, "y": b, "S": tuple(S),
                                  "opens": first and len(nb) > level})
                    first = False
    return tasks


class ResidualCache:
    """Residual of data[:, target] on S, with designs cached per S."""

    def __init__(self, data):
        self.data = data
        self.designs = {}
        self.residuals = {}
        self.infos = {}

    def prepared(self, S):
        S = tuple(S)
        if S not in self.designs:
            self.designs[S] = gcv.Prepared(tprs.design(self.data, S))
        return self.designs[S]

    def residual(self, target, S):
        key = (target, tuple(S))
        if key not in self.residuals:
            if len(S) == 0:
                self.residuals[key] = self.data[:, target].copy()
            else:
                r, info = gcv.fit(self.prepared(S), self.data[:, target])
                self.residuals[key] = r
                self.infos[key] = info
        return self.residuals[key]


def ci_pvalue(cache, method, x, y, S, num_col=35, sig=1.0, perms=None):
    rx = cache.residual(x, S)
    ry = cache.residual(y, S)
    if method == "dcc.gamma":
        return stats.dcc_gamma_decision_p(rx, ry, num_col)[0]
    if method == "hsic.gamma":
        return stats.hsic_gamma(rx, ry, sig, num_col)["p_value"]
    if method == "hsic.perm":
        return stats.hsic_perm(rx, ry, perms, sig, num_col)["p_value"]
    if method == "dcc.perm":
        return stats.dcc_perm(rx, ry, perms)["p_value"]
    raise ValueError(method)


def _pcalg_key(t):
    return (t["x"], t["y"], t["S"])


def skeleton(data, alpha=0.1, method="dcc.gamma", m_max=None, num_col=35, sig=1.0,
             replicates=100, seed=None, pvalue_fn=None, edge_runner=None):
    """Run the stable skeleton; returns adjacency, pmax, sepsets, n_edgetests, trace.

    ``edge_runner(level, chains)`` (batched methods only) may evaluate a
    level's per-edge task chains elsewhere, e.g. in worker processes: chains
    is a list of task lists, one per edge in plan order, and it returns one
    list of p-values per chain, each stopping at the first p >= alpha (the
    tests of one edge after a deletion are never run).  Edges are independent
    given the level-start graph, so this is the sequential result."""
    n, p = data.shape
    if m_max is None:
        m_max = p - 2
    adj = np.ones((p, p), dtype=bool)
    np.fill_diagonal(adj, False)
    pmax = np.full((p, p), -np.inf)
    sepsets = {}
    n_edgetests = []
    trace = []
    cache = ResidualCache(data)
    stream = rng.RStream(seed) if method in ("hsic.perm", "dcc.perm") else None
    for level in range(m_max + 1):
        tasks = make_layer_plan(adj, level)
        by_edge = {}
        for i, t in enumerate(tasks):
            by_edge.setdefault(t["edge"], []).append(i)
        pvals = {}
        if stream is None and edge_runner is not None:
            edges = list(by_edge)
            results = edge_runner(level, [[tasks[i] for i in by_edge[e]] for e in edges])
            for e, ps in zip(edges, results):
                for i, pv in zip(by_edge[e], ps):
                    pvals[i] = pv
        elif stream is None:
            for edge, idx in by_edge.items():
                for i in idx:
                    t = tasks[i]
                    pv = pvalue_fn(t) if pvalue_fn else ci_pvalue(cache, method, t["x"], t["y"], t["S"], num_col, sig)
                    pvals[i] = pv
                    if pv >= alpha:
                        break
        else:
            # one task at a time in pcalg order: the smallest ready task
            pos = {e: 0 for e in by_edge}
            while True:
                ready = [(e, by_edge[e][pos[e]]) for e in by_edge if pos[e] is not None and pos[e] < len(by_edge[e])]
                if not ready:
                    break
                e, i = min(ready, key=lambda ei: _pcalg_key(tasks[ei[1]]))
                t = tasks[i]
                if method == "hsic.perm":
                    perms = rng.hsic_permutations(stream, n, replicates)
                else:
                    perms = rng.dcc_permutations(stream, n, replicates)
                pv = ci_pvalue(cache, method, t["x"], t["y"], t["S"], num_col, sig, perms)
                pvals[i] = pv
                pos[e] = None if pv >= alpha else pos[e] + 1
        done = True
        deleted = []
        count = 0
        for i, t in enumerate(tasks):
            if i not in pvals:
                continue
            count += 1
            pv = pvals[i]
            x, y = t["edge"]
            if pv > pmax[x, y]:
                pmax[x, y] = pmax[y, x] = pv
            dele = pv >= alpha
            if dele:
                sepsets[(x, y)] = sepsets[(y, x)] = list(t["S"])
                deleted.append((x, y))
            if t["opens"]:
                done = False
            trace.append({"level": level, "x": t["x"], "y": t["y"], "S": list(t["S"]),
                          "p_value": pv, "deletes_edge": dele})
        for x, y in deleted:
            adj[x, y] = adj[y, x] = False
        n_edgetests.append(count)
        if done:
            break
    return {"adjacency": adj, "pmax": pmax, "sepsets": sepsets,
            "n_edgetests": np.array(n_edgetests), "trace": trace, "cache": cache}
