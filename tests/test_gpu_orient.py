"""WAN-PDAG orientation on the device against the oracle's (B200).

Every case of ``tests/golden/orient_oracle.npz`` (``make_orient_fixture.py``):
the oracle skeletons of the 351 x 48 SEM (seed 537) and of the 200 x 10 SEM
(seed 1), the reference's 500 x 50 development dataset with its own
skeleton, and the collider-free inputs of ``workloads.ORIENTATION_CASES``,
each for hsic.gamma and dcc.gamma.  Bars: the PDAG, the orientation counts
and the CI trace's calls and decisions exact; its p-values within 1e-9 (the
measured maximum is printed).  The full strict pipeline (device skeleton,
then device orientation) on the 351 x 48 SEM reproduces the oracle's PDAG.
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from tests.conftest import golden_path
from tests.test_orient import COUNT_KEYS, LIB_COUNT_KEYS, case_input, fixture_sepsets, fixture_trace

pytestmark = pytest.mark.gpu

CASES = [f"{c}_{m}" for c in ("skel351x48_s537", "skel200x10_s1", "dev500x50", "free300x12_s2", "free351x24_s4")
         for m in ("hsic_gamma", "dcc_gamma")]


@pytest.fixture(scope="module")
def ofx():
    with np.load(golden_path("orient_oracle.npz")) as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize("case", CASES)
def test_orientation_matches_oracle(lib_built, ofx, case):
    key = case + "_"
    method = case.rsplit("_", 2)[-2] + "." + case.rsplit("_", 1)[-1]
    X = case_input(case)
    skel = {"adjacency": ofx[key + "adjacency"], "sepsets": fixture_sepsets(ofx[key + "sepsets"])}
    out = fk.orient_wanpdag(skel, X, alpha=0.1, numCol=35, ci_method=method)
    assert np.array_equal(out["pdag"], ofx[key + "pdag"])
    d = out["diagnostics"]
    assert [d[k] for k in LIB_COUNT_KEYS] == [int(v) for v in ofx[key + "counts"]]
    assert d["residual_fits"] + d["residual_cache_hits"] == d["regrvonps_calls"]
    want = fixture_trace(ofx, key)
    t = out["ci_trace"]
    assert len(t["target"]) == len(want)
    for k, r in enumerate(want):
        assert (int(t["reverse"][k]), int(t["target"][k]), int(t["other"][k])) == \
            (r["reverse"], r["target"], r["other"]), k
        assert t["subset"][k] == r["S"] and t["residual_conditioning_set"][k] == r["Z"], k
        assert bool(t["rejected"][k]) == r["rejected"], k
    perr = float(np.max(np.abs(t["p_value"] - np.array([r["p"] for r in want])))) if want else 0.0
    print(json.dumps({"case": case, "tests": len(want), "regrvonps_calls": d["regrvonps_calls"],
                      "residual_fits": d["residual_fits"], "p_abs_err_max": perr,
                      "elapsed_sec": d["orientation_elapsed_sec"]}))
    assert perr <= 1e-9


@pytest.mark.parametrize("method", ["hsic.gamma", "dcc.gamma"])
def test_strict_wanpdag_pipeline_351x48(lib_built, ofx, method):
    X = workloads.skeleton_351x48(537)
    out = fk.fastkpc_compatible_cuda_wanpdag(X, 0.1, options={"numCol": 35, "ci_method": method})
    key = "skel351x48_s537_" + method.replace(".", "_") + "_"
    assert np.array_equal(out["skeleton"]["adjacency"], ofx[key + "adjacency"])
    assert np.array_equal(out["orientation"]["pdag"], ofx[key + "pdag"])
    m = out["metrics"]
    assert m["orientation_ci_test_count"] == len(ofx[key + "p"])
    assert m["directed_edge_count"] + m["undirected_edge_count"] == m["skeleton_edge_count"]
    print(json.dumps({"method": method, "timings": out["timings"], "metrics": m}))

