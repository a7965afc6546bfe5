"""Oracle skeletons of the n = 351, p = 48 SEM (test fixture generator).

    python tests/golden/make_skeleton_fixture.py [--seed 537] [--procs 8]

Runs the CPU oracle's default-Inf skeleton (``oracle.skeleton.skeleton``,
alpha 0.1, numCol 35, hsic sig 1) on ``fastkpc_b200.workloads.skeleton_351x48``
for hsic.gamma and then dcc.gamma, and writes
``skeleton351x48_s<seed>_oracle.npz`` beside this script: per method the
adjacency, n.edgetests, the sepsets (as a p x p x max|S| array, -1 padded),
pMax, and the logical trace in replay order (level, x, y, S, p, deleting).

Seed 537 is the deepest skeleton of seeds 1..800 under the rule of
``workloads.deep_skeleton_seed`` (it runs level 7).  Each level's per-edge
task chains are spread over spawned processes (one BLAS thread each); a
chain still runs in plan order and stops at its first deletion, so the
result is the sequential skeleton's.
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

for _var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_var] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ALPHA = 0.1
SMAX = 12

_X = None
_CACHE = None


def _init(X):
    global _X, _CACHE
    sys.path.insert(0, ROOT)
    from oracle import skeleton
    _X = X
    _CACHE = skeleton.ResidualCache(X)


def _chain(payload):
    """p-values of one edge's tasks in plan order, up to the first deletion."""
    from oracle import skeleton
    method, tasks = payload
    out = []
    for t in tasks:
        pv = skeleton.ci_pvalue(_CACHE, method, t["x"], t["y"], t["S"], 35, 1.0)
        out.append(pv)
        if pv >= ALPHA:
            break
    if len(_CACHE.designs) > 400:  # bound the worker's memory across levels
        _CACHE.designs.clear()
        _CACHE.residuals.clear()
    return out


def run(X, method, pool):
    sys.path.insert(0, ROOT)
    from oracle import skeleton

    def edge_runner(level, chains):
        # longest chains first, so the pool's last tasks are short ones
        order = sorted(range(len(chains)), key=lambda i: -len(chains[i]) * (level + 1))
        res = pool.map(_chain, [(method, chains[i]) for i in order], chunksize=1)
        out = [None] * len(chains)
        for i, r in zip(order, res):
            out[i] = r
        return out
    return skeleton.skeleton(X, ALPHA, method=method, num_col=35, sig=1.0, edge_runner=edge_runner)


def pack(res, p):
    adj = res["adjacency"].astype(bool)
    sep = np.full((p, p, SMAX), -1, dtype=np.int16)
    for (a, b), S in res["sepsets"].items():
        sep[a, b, :len(S)] = S
    tr = res["trace"]
    ts = np.full((len(tr), SMAX), -1, dtype=np.int16)
    for k, t in enumerate(tr):
        ts[k, :len(t["S"])] = t["S"]
    return {"adjacency": adj, "n_edgetests": np.asarray(res["n_edgetests"], dtype=np.int64), "sepsets": sep,
            "pmax": res["pmax"], "trace_level": np.array([t["level"] for t in tr], dtype=np.int16),
            "trace_x": np.array([t["x"] for t in tr], dtype=np.int16),
            "trace_y": np.array([t["y"] for t in tr], dtype=np.int16), "trace_S": ts,
            "trace_p": np.array([t["p_value"] for t in tr]),
            "trace_deletes": np.array([t["deletes_edge"] for t in tr], dtype=bool)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seed", type=int, default=537)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args(argv)
    sys.path.insert(0, ROOT)
    from fastkpc_b200 import workloads
    X = workloads.skeleton_351x48(args.seed)
    out = {}
    with mp.get_context("spawn").Pool(args.procs, initializer=_init, initargs=(X,)) as pool:
        for method in ("hsic.gamma", "dcc.gamma"):
            t0 = time.time()
            res = run(X, method, pool)
            print(f"{method}: n.edgetests {list(res['n_edgetests'])}, {time.time() - t0:.1f} s", flush=True)
            for k, v in pack(res, X.shape[1]).items():
                out[f"{method.replace('.', '_')}_{k}"] = v
    path = os.path.join(HERE, f"skeleton351x48_s{args.seed}_oracle.npz")
    np.savez_compressed(path, seed=np.int64(args.seed), **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
