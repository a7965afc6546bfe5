"""The 351 x 48 default-Inf skeleton against the oracle's (B200).

Data: ``workloads.skeleton_351x48(537)``, the deepest skeleton of seeds
1..800 under ``workloads.deep_skeleton_seed`` (levels 0..7 for dcc.gamma).
The oracle's skeletons for hsic.gamma and dcc.gamma come from the committed
fixture ``tests/golden/skeleton351x48_s537_oracle.npz``
(``make_skeleton_fixture.py``).  Bars: adjacency, sepsets, n.edgetests and
the logical trace -- every (level, x, y, S) in replay order and its deletion
decision -- exact; the trace's p-values and pMax within 1e-9 (the measured
maximum is printed).
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from tests.conftest import golden_path

pytestmark = pytest.mark.gpu

SEED = 537


@pytest.fixture(scope="module")
def fx():
    with np.load(golden_path(f"skeleton351x48_s{SEED}_oracle.npz")) as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize("method", ["hsic.gamma", "dcc.gamma"])
def test_skeleton_351x48_matches_oracle(lib_built, fx, method):
    key = method.replace(".", "_") + "_"
    X = workloads.skeleton_351x48(SEED)
    out = fk.fastkpc_compatible_cuda_skeleton(X, 0.1, options={"numCol": 35, "trace_level": "logical",
                                                               "ci_method": method})
    p = X.shape[1]
    assert out["n_edgetests"] == [int(v) for v in fx[key + "n_edgetests"]]
    assert np.array_equal(out["adjacency"], fx[key + "adjacency"])
    sep = fx[key + "sepsets"]
    for a in range(p):
        for b in range(p):
            want = [int(v) for v in sep[a, b] if v >= 0]
            got = out["sepsets"][a][b]
            if out["adjacency"][a, b] or a == b:
                assert got is None
            elif want or got is not None:
                assert got == want, (a, b, got, want)
    t = out["tasks"]
    n = len(fx[key + "trace_p"])
    assert len(t["level"]) == n
    assert np.array_equal(np.asarray(t["level"]), fx[key + "trace_level"])
    assert np.array_equal(np.asarray(t["x"]), fx[key + "trace_x"])
    assert np.array_equal(np.asarray(t["y"]), fx[key + "trace_y"])
    for k in range(n):
        assert list(t["S"][k]) == [int(v) for v in fx[key + "trace_S"][k] if v >= 0], k
    assert np.array_equal(np.asarray(t["native_edge_deleted"]), fx[key + "trace_deletes"])
    perr = float(np.max(np.abs(np.asarray(t["p_used"]) - fx[key + "trace_p"])))
    off = ~np.eye(p, dtype=bool)
    tested = np.isfinite(fx[key + "pmax"]) & off
    assert np.array_equal(np.isfinite(out["pMax"]) & off, tested)
    pmax_err = float(np.max(np.abs(out["pMax"][tested] - fx[key + "pmax"][tested])))
    print(json.dumps({"method": method, "logical_tests": n, "max_level": len(out["n_edgetests"]) - 1,
                      "trace_p_abs_err_max": perr, "pmax_abs_err_max": pmax_err}))
    assert perr <= 1e-9 and pmax_err <= 1e-9
