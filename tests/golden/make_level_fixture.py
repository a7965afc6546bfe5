"""Oracle records for the whole 500 x 50 level batch (test fixture generator).

    python tests/golden/make_level_fixture.py [--count 4096] [--procs 8]

Runs the CPU oracle (``oracle/``) over every triple of the single-level CI
batch -- n = 500, p = 50 nonlinear SEM (edge prob 0.08, seed 2), 4096 (x, y,
S) triples with |S| uniform on 0..4 (``fastkpc_b200.workloads``) -- and writes
``level500x50_oracle.npz`` beside this script:

* per triple: the dcc.gamma decision p, exact-screen p / statistic / mean /
  variance, the guard-band flag and (guarded triples) the low-rank statistic,
  mean and variance; the hsic.gamma (sig = 1, numCol = 35) p, statistic,
  mean and variance;
* per distinct (target, S) fit with |S| >= 1: the selected log smoothing
  parameters, the number of GCV evaluations, |r|^2 and the projections
  r . z_k on four fixed N(0, I) vectors z_k (seed 12345); the full residual
  vector for every 20th fit (in (|S|, S, target) order).

The oracle takes about a minute on 8 cores, so the GPU parity test reads
this file instead of re-running it.  Work is split by conditioning set over
spawned processes (one BLAS thread each), so each design is built once.
"""
import argparse
import multiprocessing as mp
import os
import sys
import time

# one BLAS thread per process, set before numpy loads (spawned workers import
# this module first): the pool supplies the parallelism
for _var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_var] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "level500x50_oracle.npz")
PROJ_SEED = 12345
FULL_EVERY = 20
SMAX = 4


def _worker(payload):
    sys.path.insert(0, ROOT)
    from oracle import skeleton, stats
    X, groups = payload
    cache = skeleton.ResidualCache(X)
    fits, recs = {}, {}
    for S, targets, tests in groups:
        for t in targets:
            r = cache.residual(t, S)
            info = cache.infos.get((t, tuple(S)))
            fits[(t, tuple(S))] = (r, np.asarray(info["log_sp"], dtype=np.float64), int(info["calls"]))
        for k, x, y in tests:
            rx, ry = cache.residual(x, S), cache.residual(y, S)
            ex = stats.dcov_gamma_exact(rx, ry)
            p_dec, p_ex, guarded = stats.dcc_gamma_decision_p(rx, ry, 35)
            lg = stats.dcov_gamma_legacy(rx, ry, 35) if guarded else None
            hs = stats.hsic_gamma(rx, ry, 1.0, 35)
            recs[k] = (p_dec, p_ex, guarded, ex, lg, hs)
        cache.residuals.clear()  # the next set's fits share nothing with these
        cache.designs.clear()
    return fits, recs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args(argv)
    sys.path.insert(0, ROOT)
    from fastkpc_b200 import workloads
    X, triples = workloads.level_batch_500x50(count=args.count)
    n = X.shape[0]

    by_set = {}
    for k, (x, y, S) in enumerate(triples):
        S = tuple(sorted(S))
        g = by_set.setdefault(S, [set(), []])
        g[0].update((x, y))
        g[1].append((k, x, y))
    # largest designs first, dealt to the least-loaded worker
    cost = {S: (1 + 9 * len(S)) ** 2 * len(g[0]) if len(S) > 2 else 900 * len(g[0]) for S, g in by_set.items()}
    load = [0.0] * args.procs
    work = [[] for _ in range(args.procs)]
    for S in sorted(by_set, key=lambda s: -cost[s]):
        w = min(range(args.procs), key=lambda i: load[i])
        load[w] += cost[S]
        work[w].append((list(S), sorted(by_set[S][0]) if S else [], by_set[S][1]))
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.procs) as pool:
        parts = pool.map(_worker, [(X, w) for w in work if w])
    fits, recs = {}, {}
    for f, r in parts:
        fits.update(f)
        recs.update(r)
    print(f"oracle: {len(recs)} triples, {len(fits)} fits in {time.time() - t0:.1f} s")

    count = len(triples)
    tx = np.array([t[0] for t in triples], dtype=np.int32)
    ty = np.array([t[1] for t in triples], dtype=np.int32)
    ts = np.full((count, SMAX), -1, dtype=np.int32)
    for k, (_, _, S) in enumerate(triples):
        ts[k, :len(S)] = sorted(S)
    cols = {name: np.zeros(count) for name in (
        "dcc_p", "dcc_p_exact", "dcc_stat_exact", "dcc_mean_exact", "dcc_var_exact",
        "dcc_stat_lowrank", "dcc_mean_lowrank", "dcc_var_lowrank",
        "hsic_p", "hsic_stat", "hsic_mean", "hsic_var")}
    guarded = np.zeros(count, dtype=bool)
    for k in range(count):
        p_dec, p_ex, g, ex, lg, hs = recs[k]
        cols["dcc_p"][k], cols["dcc_p_exact"][k] = p_dec, p_ex
        cols["dcc_stat_exact"][k], cols["dcc_mean_exact"][k], cols["dcc_var_exact"][k] = (
            ex["statistic"], ex["mean"], ex["variance"])
        guarded[k] = g
        if g:
            cols["dcc_stat_lowrank"][k], cols["dcc_mean_lowrank"][k], cols["dcc_var_lowrank"][k] = (
                lg["statistic"], lg["mean"], lg["variance"])
        else:
            for c in ("dcc_stat_lowrank", "dcc_mean_lowrank", "dcc_var_lowrank"):
                cols[c][k] = np.nan
        cols["hsic_p"][k], cols["hsic_stat"][k], cols["hsic_mean"][k], cols["hsic_var"][k] = (
            hs["p_value"], hs["statistic"], hs["mean"], hs["variance"])

    keys = sorted((k for k in fits if len(k[1]) > 0), key=lambda k: (len(k[1]), k[1], k[0]))
    nf = len(keys)
    z = np.random.default_rng(PROJ_SEED).standard_normal((4, n))
    f_target = np.array([k[0] for k in keys], dtype=np.int32)
    f_set = np.full((nf, SMAX), -1, dtype=np.int32)
    f_logsp = np.full((nf, SMAX), np.nan)
    f_calls = np.zeros(nf, dtype=np.int32)
    f_norm2 = np.zeros(nf)
    f_proj = np.zeros((nf, 4))
    full_idx = np.arange(0, nf, FULL_EVERY, dtype=np.int32)
    full = np.zeros((n, len(full_idx)), order="F")
    for i, key in enumerate(keys):
        r, lsp, calls = fits[key]
        f_set[i, :len(key[1])] = key[1]
        f_logsp[i, :len(lsp)] = lsp
        f_calls[i] = calls
        f_norm2[i] = float(r @ r)
        f_proj[i] = z @ r
    for j, i in enumerate(full_idx):
        full[:, j] = fits[keys[i]][0]
    np.savez_compressed(args.out, x=tx, y=ty, S=ts, guarded=guarded, fit_target=f_target, fit_S=f_set,
                        fit_log_sp=f_logsp, fit_calls=f_calls, fit_norm2=f_norm2, fit_proj=f_proj,
                        full_index=full_idx, full_residuals=full, proj_seed=np.int64(PROJ_SEED), **cols)
    print(f"wrote {args.out} ({os.path.getsize(args.out) / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
