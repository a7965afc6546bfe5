"""Oracle WAN-PDAG orientations (test fixture generator).

    python tests/golden/make_orient_fixture.py

Runs the CPU oracle's orientation (``oracle.orient.orient``, alpha 0.1,
numCol 35, hsic sig 1) on

* the oracle skeletons of ``skeleton351x48_s537_oracle.npz`` (the 351 x 48
  SEM of seed 537), for hsic.gamma and dcc.gamma;
* the oracle skeleton of ``workloads.skeleton_200x10(1)`` (computed here),
  for both methods;
* the reference's own 500 x 50 development dataset and its dcc.gamma
  skeleton (``dev500x50.npz`` and the sepsets of ``dev500x50_trace.json``,
  read from the reference's fixture by ``make_golden.py``), for both methods;
* the collider-free inputs ``workloads.ORIENTATION_CASES`` (every
  neighbourhood goes through regrVonPS), for both methods;

and writes ``orient_oracle.npz`` beside this script: per case and method the
input adjacency and sepsets (p x p x max|S|, -1 padded), the PDAG, the counts
(collider, rule1, rule2, rule3, generalized, regrVonPS calls) and the CI
trace in call order (reverse flag, target, other, S and Z -1 padded, p,
rejected).
"""
import json
import os
import sys
import time

for _var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ[_var] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ALPHA = 0.1
SMAX = 48
COUNT_KEYS = ("collider", "rule1", "rule2", "rule3", "generalized", "regrvonps_calls")


def pad_sets(sets, width):
    out = np.full((len(sets), width), -1, dtype=np.int16)
    for k, s in enumerate(sets):
        out[k, :len(s)] = s
    return out


def sepset_array(sepsets, p):
    sep = np.full((p, p, SMAX), -1, dtype=np.int16)
    for (a, b), S in sepsets.items():
        sep[a, b, :len(S)] = S
    return sep


def sepset_dict(sep):
    p = sep.shape[0]
    return {(a, b): [int(v) for v in sep[a, b] if v >= 0] for a in range(p) for b in range(p)
            if np.any(sep[a, b] >= 0)}


def run_case(out, name, X, adj, sepsets, method):
    from oracle import orient
    t0 = time.time()
    pdag, trace, counts = orient.orient(X, adj, sepsets, method, ALPHA, 35, 1.0)
    key = f"{name}_{method.replace('.', '_')}_"
    p = X.shape[1]
    out[key + "adjacency"] = np.asarray(adj, dtype=bool)
    out[key + "sepsets"] = sepset_array(sepsets, p)
    out[key + "pdag"] = pdag.astype(np.int8)
    out[key + "counts"] = np.array([counts[k] for k in COUNT_KEYS], dtype=np.int64)
    out[key + "reverse"] = np.array([t["reverse"] for t in trace], dtype=np.int8)
    out[key + "target"] = np.array([t["target"] for t in trace], dtype=np.int16)
    out[key + "other"] = np.array([t["other"] for t in trace], dtype=np.int16)
    out[key + "S"] = pad_sets([t["S"] for t in trace], p)
    out[key + "Z"] = pad_sets([t["Z"] for t in trace], p)
    out[key + "p"] = np.array([t["p"] for t in trace])
    out[key + "rejected"] = np.array([t["rejected"] for t in trace], dtype=bool)
    print(f"{name} {method}: {counts}, {len(trace)} tests, {time.time() - t0:.1f} s", flush=True)


def main():
    sys.path.insert(0, ROOT)
    from fastkpc_b200 import workloads
    from oracle import skeleton
    out = {}
    X = workloads.skeleton_351x48(537)
    with np.load(os.path.join(HERE, "skeleton351x48_s537_oracle.npz")) as f:
        for method in ("hsic.gamma", "dcc.gamma"):
            k = method.replace(".", "_") + "_"
            run_case(out, "skel351x48_s537", X, f[k + "adjacency"], sepset_dict(f[k + "sepsets"]), method)
    X = workloads.skeleton_200x10(1)
    for method in ("hsic.gamma", "dcc.gamma"):
        res = skeleton.skeleton(X, ALPHA, method=method, num_col=35, sig=1.0)
        run_case(out, "skel200x10_s1", X, res["adjacency"], res["sepsets"], method)
    X = np.load(os.path.join(HERE, "dev500x50.npz"))["data"]
    adj = np.load(os.path.join(HERE, "dev500x50.npz"))["adjacency"].astype(bool)
    with open(os.path.join(HERE, "dev500x50_trace.json")) as f:
        sepsets = {(i, j): S for i, j, S in json.load(f)["sepsets"]}
    for method in ("hsic.gamma", "dcc.gamma"):
        run_case(out, "dev500x50", X, adj, sepsets, method)
    for name, kw in workloads.ORIENTATION_CASES.items():
        X, adj, sepsets = workloads.orientation_collider_free(**kw)
        for method in ("hsic.gamma", "dcc.gamma"):
            run_case(out, name, X, adj, sepsets, method)
    path = os.path.join(HERE, "orient_oracle.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.3f} MB)")


if __name__ == "__main__":
    main()
