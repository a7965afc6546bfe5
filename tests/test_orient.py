"""WAN-PDAG orientation on the CPU: the oracle's rules on hand-built graphs,
the library's graph logic (``fkpc_orient_wanpdag_custom``, no device)
against the oracle's with the same CI answers, and the fixture pin.

The library's orientation takes its CI answers from an evaluator; here the
evaluator is either a deterministic stub (p-values hashed from the call) or
the oracle's own regrVonPS, so pdag, counts and the CI trace must agree
exactly.
"""
import hashlib

import numpy as np
import pytest
from threadpoolctl import threadpool_limits

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from oracle import orient
from tests.conftest import golden_path

COUNT_KEYS = ("collider", "rule1", "rule2", "rule3", "generalized", "regrvonps_calls")
LIB_COUNT_KEYS = ("collider_orientations", "rule1_orientations", "rule2_orientations", "rule3_orientations",
                  "generalized_orientations", "regrvonps_calls")


def graph(p, directed=(), undirected=()):
    g = np.zeros((p, p), dtype=np.int64)
    for a, b in directed:
        g[a, b] = 1
    for a, b in undirected:
        g[a, b] = g[b, a] = 1
    return g


def test_rule1_orients_away_from_an_arrow():
    g = graph(3, directed=[(0, 1)], undirected=[(1, 2)])
    assert orient.rule1(g) == 1
    assert g[1, 2] == 1 and g[2, 1] == 0
    g = graph(3, directed=[(0, 1)], undirected=[(1, 2), (0, 2)])  # 0 and 2 adjacent: no rule-1 step
    assert orient.rule1(g) == 0 and g[1, 2] == 1 and g[2, 1] == 1


def test_rule2_follows_a_directed_chain():
    g = graph(3, directed=[(0, 2), (2, 1)], undirected=[(0, 1)])
    assert orient.rule2(g) == 1
    assert g[0, 1] == 1 and g[1, 0] == 0


def test_rule3_two_non_adjacent_parents():
    # a = 0, b = 1, c1 = 2, c2 = 3: 0 - 2 -> 1, 0 - 3 -> 1, 0 - 1, 2 and 3 non-adjacent
    g = graph(4, directed=[(2, 1), (3, 1)], undirected=[(0, 1), (0, 2), (0, 3)])
    assert orient.rule3(g) == 1
    assert g[0, 1] == 1 and g[1, 0] == 0
    g = graph(4, directed=[(2, 1), (3, 1)], undirected=[(0, 1), (0, 2), (0, 3), (2, 3)])
    assert orient.rule3(g) == 0


def test_check_immor():
    g = graph(4, directed=[(3, 0)], undirected=[(0, 1), (0, 2)])
    assert not orient.check_immor(g, 0, [1])        # parent 3 and 1 non-adjacent
    g[3, 1] = g[1, 3] = 1
    assert orient.check_immor(g, 0, [1])
    assert not orient.check_immor(g, 0, [1, 2])     # 1 and 2 non-adjacent
    g[1, 2] = g[2, 1] = 1
    g[3, 2] = g[2, 3] = 1
    assert orient.check_immor(g, 0, [1, 2])


def _stub(table=None, default=0.5):
    """p-values of a regrVonPS call: table[(target, tuple(S))] (one per member), else ``default``."""
    def pvals(target, S, Z):
        if table is not None and (target, tuple(S)) in table:
            return list(table[(target, tuple(S))])
        return [default] * len(S)
    return pvals


def _hashed(target, S, Z):
    """Deterministic pseudo-p-values of a call: a member is dependent (p < 0.1) about a third of the time."""
    out = []
    for s in S:
        h = hashlib.sha256(f"{target}|{tuple(S)}|{tuple(Z)}|{s}".encode()).digest()
        out.append(int.from_bytes(h[:8], "little") / 2.0 ** 64 * 0.3)
    return out


def oracle_with(pvals, adjacency, sepsets, alpha=0.1):
    """oracle.orient with every regrVonPS answered by ``pvals``; returns (pdag, trace, counts)."""
    trace = []

    def regress(pd, v, S, context):
        Z = sorted(list(S) + orient._parents(pd, v))
        pv = pvals(v, list(S), Z)
        for k, s in enumerate(S):
            trace.append({"reverse": context, "target": v, "other": s, "S": list(S), "Z": Z, "p": pv[k],
                          "rejected": pv[k] < alpha})
        return sum(p < alpha for p in pv)
    pdag, _, counts = orient.orient(None, adjacency, sepsets, alpha=alpha, regress=regress)
    return pdag, trace, counts


def assert_same(lib, pdag, trace, counts):
    assert np.array_equal(lib["pdag"], pdag)
    assert [lib["diagnostics"][k] for k in LIB_COUNT_KEYS] == [counts[k] for k in COUNT_KEYS]
    t = lib["ci_trace"]
    assert len(t["target"]) == len(trace)
    for k, row in enumerate(trace):
        assert (int(t["reverse"][k]), int(t["target"][k]), int(t["other"][k])) == \
            (row["reverse"], row["target"], row["other"]), k
        assert t["subset"][k] == list(row["S"]) and t["residual_conditioning_set"][k] == list(row["Z"]), k
        assert t["p_value"][k] == row["p"] and bool(t["rejected"][k]) == bool(row["rejected"]), k


def test_generalized_orientation_of_a_chain():
    """0 - 1 - 2 with 1 in sepset(0, 2): no collider; regrVonPS accepts 0 -> 1
    (1's residual on 0 is independent of 0, 0's residual on 1 is not
    independent of 1), so 1 -> 2 follows, and the rest of 1's listed
    subsets fail checkImmor."""
    adj = graph(3, undirected=[(0, 1), (1, 2)]).astype(bool)
    seps = {(0, 2): [1], (2, 0): [1]}
    pvals = _stub({(1, (0,)): [0.5]}, default=0.01)
    pdag, trace, counts = oracle_with(pvals, adj, seps)
    assert np.array_equal(pdag, graph(3, directed=[(0, 1), (1, 2)]))
    assert counts["generalized"] == 1 and counts["regrvonps_calls"] == 4
    assert [(r["reverse"], r["target"], tuple(r["S"])) for r in trace] == [(0, 0, (1,)), (0, 2, (1,)),
                                                                           (0, 1, (0,)), (1, 0, (1,))]
    lib = fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": seps}, 3, 0.1, pvals)
    assert_same(lib, pdag, trace, counts)


def test_kite_orients_by_rule3_after_an_accepted_orientation(lib_built):
    """A kite 2 -> 1 <- 3 (collider: 2, 3 non-adjacent, 1 not in sepset(2, 3))
    with 0 adjacent to 1, 2, 3, beside a chain 4 - 5 - 6.  Every regrVonPS is
    dependent except 5's on {4}, so the generalized stage accepts 4 -> 5 (and
    5 -> 6); the rules that follow orient 0 -> 1 by rule 3 (0 - 2 -> 1,
    0 - 3 -> 1, 2 and 3 non-adjacent); 0 - 2 and 0 - 3 stay undirected."""
    adj = graph(7, undirected=[(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (4, 5), (5, 6)]).astype(bool)
    seps = {(2, 3): [0], (3, 2): [0], (4, 6): [5], (6, 4): [5]}
    pvals = _stub({(5, (4,)): [0.5]}, default=0.01)
    pdag, trace, counts = oracle_with(pvals, adj, seps)
    want = graph(7, directed=[(2, 1), (3, 1), (0, 1), (4, 5), (5, 6)], undirected=[(0, 2), (0, 3)])
    assert np.array_equal(pdag, want)
    assert counts == {"collider": 1, "rule1": 0, "rule2": 0, "rule3": 1, "generalized": 1, "regrvonps_calls": 7}
    lib = fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": seps}, 7, 0.1, pvals)
    assert_same(lib, pdag, trace, counts)


def test_colliders_and_empty_graph(lib_built):
    adj = graph(3, undirected=[(0, 1), (1, 2)]).astype(bool)
    lib = fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": {(0, 2): [], (2, 0): []}}, 3, 0.1, _stub())
    assert np.array_equal(lib["pdag"], graph(3, directed=[(0, 1), (2, 1)]))
    # (0, 1, 2) orients both edges; (2, 1, 0) finds them oriented and changes nothing
    assert lib["diagnostics"]["collider_orientations"] == 1 and lib["diagnostics"]["regrvonps_calls"] == 0
    lib = fk.orient_wanpdag_custom({"adjacency": np.zeros((4, 4), bool), "sepsets": None}, 4, 0.1, _stub())
    assert not lib["pdag"].any() and lib["diagnostics"]["ci_test_count"] == 0


@pytest.mark.parametrize("seed", range(60))
def test_library_graph_logic_matches_oracle_on_random_skeletons(lib_built, seed):
    """Random skeletons (most non-adjacent pairs separated by all other nodes,
    so the generalized stage and the rules run; 60 seeds give about 300
    collider, 260 rule-1, 90 rule-2 and 70 generalized orientations over
    1100 regrVonPS calls) with hashed p-values."""
    rs = np.random.default_rng(1000 + seed)
    p = int(rs.integers(4, 13))
    upper = np.triu(rs.random((p, p)) < rs.uniform(0.25, 0.7), 1)
    adj = upper | upper.T
    seps = {}
    for a in range(p):
        for b in range(a + 1, p):
            if not adj[a, b]:
                others = [c for c in range(p) if c not in (a, b)]
                if rs.random() < 0.75:
                    S = others
                else:
                    S = sorted(rs.choice(others, size=int(rs.integers(0, min(3, len(others)) + 1)),
                                         replace=False).tolist())
                seps[(a, b)] = S
                seps[(b, a)] = S
    pdag, trace, counts = oracle_with(_hashed, adj, seps)
    lib = fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": seps}, p, 0.1, _hashed)
    assert_same(lib, pdag, trace, counts)


def test_custom_evaluator_errors_propagate(lib_built):
    adj = graph(3, undirected=[(0, 1), (1, 2)]).astype(bool)

    def bad(target, S, Z):
        raise RuntimeError("backend down")
    with pytest.raises(RuntimeError, match="backend down"):
        fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": {(0, 2): [1]}}, 3, 0.1, bad)
    with pytest.raises(fk.FkpcError):
        fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": {(0, 2): [1]}}, 3, 0.1, lambda t, S, Z: [float("nan")])
    asym = adj.copy()
    asym[0, 1] = False
    with pytest.raises(fk.FkpcError, match="symmetric"):
        fk.orient_wanpdag_custom({"adjacency": asym, "sepsets": None}, 3, 0.1, _stub())


@pytest.fixture(scope="module")
def ofx():
    with np.load(golden_path("orient_oracle.npz")) as f:
        return {k: f[k] for k in f.files}


def fixture_cases(ofx):
    names = sorted({k.rsplit("_gamma_", 1)[0] + "_gamma" for k in ofx if k.endswith("_pdag")})
    return names


def case_input(name):
    """(X, adjacency, sepsets) of a fixture case, rebuilt from the workload generators."""
    if name.startswith("skel351x48_s537"):
        return workloads.skeleton_351x48(537)
    if name.startswith("skel200x10_s1"):
        return workloads.skeleton_200x10(1)
    if name.startswith("dev500x50"):
        return np.load(golden_path("dev500x50.npz"))["data"]
    for case, kw in workloads.ORIENTATION_CASES.items():
        if name.startswith(case):
            return workloads.orientation_collider_free(**kw)[0]
    raise KeyError(name)


def fixture_sepsets(sep):
    p = sep.shape[0]
    return {(a, b): [int(v) for v in sep[a, b] if v >= 0] for a in range(p) for b in range(p)
            if np.any(sep[a, b] >= 0)}


def fixture_trace(ofx, key):
    out = []
    for k in range(len(ofx[key + "p"])):
        out.append({"reverse": int(ofx[key + "reverse"][k]), "target": int(ofx[key + "target"][k]),
                    "other": int(ofx[key + "other"][k]), "S": [int(v) for v in ofx[key + "S"][k] if v >= 0],
                    "Z": [int(v) for v in ofx[key + "Z"][k] if v >= 0], "p": float(ofx[key + "p"][k]),
                    "rejected": bool(ofx[key + "rejected"][k])})
    return out


def test_fixture_covers_the_cases(ofx):
    names = fixture_cases(ofx)
    assert len(names) == 10
    total = {k: 0 for k in COUNT_KEYS}
    for name in names:
        for k, v in zip(COUNT_KEYS, ofx[name + "_counts"]):
            total[k] += int(v)
    assert total["collider"] > 0 and total["rule1"] > 0 and total["rule2"] > 0 and total["generalized"] > 0


@pytest.mark.parametrize("case", ["skel200x10_s1_dcc_gamma", "free300x12_s2_hsic_gamma", "free351x24_s4_dcc_gamma",
                                  "dev500x50_dcc_gamma"])
def test_oracle_reproduces_fixture_and_library_logic_agrees(lib_built, ofx, case):
    """The oracle regenerates the fixture (pin), and the library's graph logic
    fed the oracle's regrVonPS p-values reproduces it exactly."""
    key = case + "_"
    method = case.rsplit("_", 2)[-2] + "." + case.rsplit("_", 1)[-1]
    X = case_input(case)
    adj = ofx[key + "adjacency"]
    seps = fixture_sepsets(ofx[key + "sepsets"])
    with threadpool_limits(1):
        pdag, trace, counts = orient.orient(X, adj, seps, method, 0.1, 35, 1.0)
        assert np.array_equal(pdag, ofx[key + "pdag"])
        assert [counts[k] for k in COUNT_KEYS] == [int(v) for v in ofx[key + "counts"]]
        want = fixture_trace(ofx, key)
        assert [(r["target"], r["other"], r["S"], r["Z"], r["rejected"]) for r in trace] == \
            [(r["target"], r["other"], r["S"], r["Z"], r["rejected"]) for r in want]
        assert max((abs(a["p"] - b["p"]) for a, b in zip(trace, want)), default=0.0) <= 1e-12
        by_call = {}
        for r in want:
            by_call.setdefault((r["target"], tuple(r["S"]), tuple(r["Z"])), []).append(r["p"])

        def replay(target, S, Z):  # a repeated call repeats its p-values
            return by_call[(target, tuple(S), tuple(Z))][:len(S)]
        lib = fk.orient_wanpdag_custom({"adjacency": adj, "sepsets": seps}, X.shape[1], 0.1, replay)
    assert_same(lib, ofx[key + "pdag"], want, dict(zip(COUNT_KEYS, (int(v) for v in ofx[key + "counts"]))))


def test_orientation_rejects_permutation_methods_and_other_settings():
    X = workloads.skeleton_200x10(1)
    skel = {"adjacency": np.zeros((10, 10), bool), "sepsets": None}
    with pytest.raises(ValueError):
        fk.orient_wanpdag(skel, X, ci_method="dcc.perm")
    with pytest.raises(ValueError):
        fk.orient_wanpdag(skel, X, solve_confl=True)
    with pytest.raises(ValueError):
        fk.fastkpc_compatible_cuda_wanpdag(X, 0.1, options={"trace_level": "summary"})
