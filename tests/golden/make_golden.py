"""Regenerate the golden fixtures in this directory from the reference tree.

Run from the repository root with the reference checkout available:

    python tests/golden/make_golden.py /path/to/reference

It reads two ``.rds`` fixtures the reference commits under
``fastkpc/tests/fixtures/`` and writes plain files the test-suite loads:

* ``dev500x50.npz`` -- the 500x50 development dataset (seed 1050050, generator
  ``fastkpc/R/full_cuda_ci_phase10_development_500x50.R:14-47``) and the
  reference's dcc.gamma default-Inf skeleton outcome: adjacency, pMax,
  n.edgetests.
* ``dev500x50_trace.json`` -- the 2722-row logical trace (level, x, y, S,
  p-value, deletes_edge), the deletion trace and the sepsets, all 0-based.
* ``legacy_dcov_gamma.json`` -- residual pairs with kpcalg ``dcov.gamma``
  p-value, nV2, mean and variance (``fastkpc/tests/test_legacy_dcov_gamma_cpp_oracle.R:16-47``).
"""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from rds_reader import read_rds  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def _s_list(key):
    return [] if key in ("", None) else [int(v) - 1 for v in key.split("|")]


def dev500x50(ref):
    path = os.path.join(ref, "fastkpc/tests/fixtures/full_cuda_ci_development_500x50_v2.rds")
    o = read_rds(path)
    data = o["data"]
    n, p = (int(v) for v in data.attrs["dim"].value)
    X = np.asarray(data.value, dtype=np.float64).reshape(p, n).T.copy()
    ref_out = o["oracle"]["reference"]
    adj = np.asarray(ref_out["adjacency"].value).reshape(p, p).T.astype(np.int8)
    pmax = np.asarray(ref_out["pMax"].value, dtype=np.float64).reshape(p, p).T.copy()
    ntests = np.asarray(ref_out["n.edgetests"].value, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "dev500x50.npz"), data=X, adjacency=adj,
                        pmax=pmax, n_edgetests=ntests,
                        baseline_elapsed_sec=np.float64(o["baseline_elapsed_sec"].value[0]))

    lt = o["oracle"]["logical_trace"]
    rows = []
    for i in range(len(lt["level"].value)):
        rows.append({
            "level": int(lt["level"].value[i]),
            "x": int(lt["x"].value[i]) - 1,
            "y": int(lt["y"].value[i]) - 1,
            "S": _s_list(lt["S_key"].value[i]),
            "p_value": float(lt["p_value"].value[i]),
            "deletes_edge": bool(lt["deletes_edge"].value[i]),
        })
    dt = o["oracle"]["deletion_trace"]
    deletions = []
    for i in range(len(dt["level"].value)):
        deletions.append({
            "level": int(dt["level"].value[i]),
            "edge_x": int(dt["edge_x"].value[i]) - 1,
            "edge_y": int(dt["edge_y"].value[i]) - 1,
            "x": int(dt["tested_x"].value[i]) - 1,
            "y": int(dt["tested_y"].value[i]) - 1,
            "S": _s_list(dt["S_key"].value[i]),
            "p_value": float(dt["p_value"].value[i]),
        })
    sepsets = []
    ss = ref_out["sepsets"]
    for i, row in enumerate(ss.value):
        for j, cell in enumerate(row.value):
            if cell is not None and len(cell.value) > 0:
                sepsets.append([i, j, sorted(int(v) - 1 for v in cell.value)])
    with open(os.path.join(HERE, "dev500x50_trace.json"), "w") as f:
        json.dump({"n": n, "p": p, "alpha": 0.1, "num_col": 35, "ci_method": "dcc.gamma",
                   "logical_trace": rows, "deletion_trace": deletions, "sepsets": sepsets},
                  f, separators=(",", ":"))


def legacy_dcov(ref):
    path = os.path.join(ref, "fastkpc/tests/fixtures/legacy_dcov_gamma_oracle_v1.rds")
    cases = []
    for case in read_rds(path).value:
        meta = case["meta"]
        res = case["residuals"]
        cases.append({
            "case_id": meta["case_id"].value[0],
            "num_col": int(meta["numCol"].value[0]),
            "alpha": float(meta["alpha"].value[0]),
            "p_value": float(meta["p.value"].value[0]),
            "delete_edge": bool(meta["delete_edge"].value[0]),
            "nV2": float(meta["nV2"].value[0]),
            "mean": float(meta["nV2Mean"].value[0]),
            "variance": float(meta["nV2Variance"].value[0]),
            "rx": [float(v) for v in res["rx"].value],
            "ry": [float(v) for v in res["ry"].value],
        })
    with open(os.path.join(HERE, "legacy_dcov_gamma.json"), "w") as f:
        json.dump({"cases": cases}, f)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    dev500x50(ref)
    legacy_dcov(ref)
    print("golden fixtures written to", HERE)
