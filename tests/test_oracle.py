"""The oracle against the reference's own golden vectors (CPU only).

Pins: the R-compatible stream against the 500x50 fixture data (its first
column is the first 500 rnorm draws after set.seed(1050050)); legacy
dcov.gamma against fastkpc/tests/fixtures/legacy_dcov_gamma_oracle_v1.rds;
the full dcc.gamma default-Inf skeleton against the 500x50 fixture
(adjacency, n.edgetests, sepsets and all 2722 decisions).
"""
import json
import math

import numpy as np
import pytest
from scipy.special import gammaincc

from oracle import gcv, rng, skeleton, stats, tprs
from tests.conftest import golden_path


def test_r_stream_reproduces_fixture_rnorm(dev500):
    s = rng.RStream(1050050)
    z = np.array([s.norm_rand() for _ in range(500)])
    # qnorm vs ndtri rounding only
    assert np.max(np.abs(z - dev500["data"][:, 0])) < 1e-13


def test_permutation_tables_are_permutations():
    s = rng.RStream(7)
    d = rng.dcc_permutations(s, 50, 5)
    h = rng.hsic_permutations(s, 50, 5)
    for t in (d, h):
        for row in t:
            assert sorted(row.tolist()) == list(range(50))
    # the dcc stream consumes exactly R (n - 1) uniforms
    s2 = rng.RStream(7)
    rng.dcc_permutations(s2, 50, 5)
    assert s2.draws == 5 * 49


@pytest.fixture(scope="module")
def legacy_cases():
    with open(golden_path("legacy_dcov_gamma.json")) as f:
        return json.load(f)["cases"]


def test_legacy_dcov_gamma_matches_reference_cases(legacy_cases):
    assert len(legacy_cases) >= 6
    for c in legacy_cases:
        r = stats.dcov_gamma_legacy(np.array(c["rx"]), np.array(c["ry"]), c["num_col"])
        assert abs(r["p_value"] - c["p_value"]) <= 1e-8, c["case_id"]
        assert abs(r["statistic"] - c["nV2"]) <= 1e-8, c["case_id"]
        assert abs(r["mean"] - c["mean"]) <= 1e-8, c["case_id"]
        assert abs(r["variance"] - c["variance"]) <= 1e-8, c["case_id"]
        assert (r["p_value"] >= c["alpha"]) == c["delete_edge"], c["case_id"]


def test_exact_dcov_matches_direct_formula():
    rs = np.random.default_rng(3)
    x, y = rs.normal(size=40), rs.normal(size=40)
    r = stats.dcov_gamma_exact(x, y)
    a = np.abs(x[:, None] - x[None, :])
    b = np.abs(y[:, None] - y[None, :])
    H = np.eye(40) - 1.0 / 40
    A, B = H @ a @ H, H @ b @ H
    assert math.isclose(r["statistic"], float(np.sum(A * B)) / 40, rel_tol=1e-12)
    assert 0.0 <= r["p_value"] <= 1.0


def test_gamma_tail_is_scipy():
    assert stats._gamma_p(2.0, 1.0, 0.5) == pytest.approx(gammaincc(2.0, 4.0), rel=1e-15)


def test_inchol_factor_reconstructs_kernel():
    rs = np.random.default_rng(5)
    r = rs.normal(size=60)
    G = stats.inchol(r, 1.0, 60, tol=1e-12)
    K = np.exp(-(r[:, None] - r[None, :]) ** 2)
    assert np.max(np.abs(G @ G.T - K)) < 1e-9


def test_tprs_design_widths(dev500):
    d = dev500["data"]
    for S, q in (([3], 10), ([3, 7], 30), ([1, 5, 9], 28), ([2, 11, 17, 40], 37)):
        des = tprs.design(d, S)
        assert des["X"].shape == (500, q)
        assert np.allclose(des["X"][:, 1:].mean(axis=0), 0.0, atol=1e-12)  # centred smooths


def test_gcv_gradient_matches_finite_differences(dev500):
    d = dev500["data"]
    prep = gcv.Prepared(tprs.design(d, [1, 5, 9]))
    rho = np.array([0.5, -1.0, 2.0])
    v, g, H = gcv.gcv_value_grad_hess(prep, d[:, 20], rho)
    h = 1e-5
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        vp, gp, _ = gcv.gcv_value_grad_hess(prep, d[:, 20], rho + e)
        vm, gm, _ = gcv.gcv_value_grad_hess(prep, d[:, 20], rho - e)
        assert (vp - vm) / (2 * h) == pytest.approx(g[j], rel=1e-6, abs=1e-10)
        assert np.allclose((gp - gm) / (2 * h), H[:, j], rtol=1e-5, atol=1e-9)


@pytest.mark.slow
def test_oracle_reproduces_500x50_dcc_gamma_skeleton(dev500, dev500_trace):
    out = skeleton.skeleton(dev500["data"], 0.1, "dcc.gamma")
    assert out["n_edgetests"].tolist() == dev500["n_edgetests"].tolist()
    assert np.array_equal(out["adjacency"].astype(np.int8), dev500["adjacency"])
    ref = {(r["level"], r["x"], r["y"], tuple(r["S"])): r for r in dev500_trace["logical_trace"]}
    assert len(out["trace"]) == len(ref)
    for row in out["trace"]:
        g = ref[(row["level"], row["x"], row["y"], tuple(row["S"]))]
        assert row["deletes_edge"] == g["deletes_edge"]
    ref_sep = {(i, j): s for i, j, s in dev500_trace["sepsets"]}
    for (i, j), s in out["sepsets"].items():
        if (i, j) in ref_sep:
            assert sorted(s) == ref_sep[(i, j)]
    assert all(((i, j) in out["sepsets"]) for (i, j) in ref_sep)


def test_level_fixture_is_the_workload_and_the_oracle():
    """The committed 500x50 level-batch fixture: its triples are the workload
    generator's, and the oracle re-run on a sample reproduces its records."""
    from threadpoolctl import threadpool_limits
    from fastkpc_b200 import workloads
    from tests.golden import level_report
    fx = level_report.load()
    X, triples = workloads.level_batch_500x50(count=len(fx["x"]))
    assert level_report.triples(fx) == triples
    cache = skeleton.ResidualCache(X)
    # the fixture was written with one BLAS thread per process; threaded BLAS
    # reductions round differently and can move magic's path in the last bits
    with threadpool_limits(limits=1):
        for k in (0, 1, 2, 100, 2048, 4095):
            x, y, S = triples[k]
            rx, ry = cache.residual(x, S), cache.residual(y, S)
            p, pe, g = stats.dcc_gamma_decision_p(rx, ry, 35)
            assert abs(p - fx["dcc_p"][k]) <= 1e-13 and abs(pe - fx["dcc_p_exact"][k]) <= 1e-13
            assert g == fx["guarded"][k]
            assert abs(stats.hsic_gamma(rx, ry, 1.0, 35)["p_value"] - fx["hsic_p"][k]) <= 1e-13
    # the report of the fixture against itself is all zeros
    g = fx["guarded"]
    rec = {"flags": g.astype(np.int64),
           "statistic": np.where(g, fx["dcc_stat_lowrank"], fx["dcc_stat_exact"]),
           "mean": np.where(g, fx["dcc_mean_lowrank"], fx["dcc_mean_exact"]),
           "variance": np.where(g, fx["dcc_var_lowrank"], fx["dcc_var_exact"]),
           "p_exact": fx["dcc_p_exact"], "p_value": fx["dcc_p"]}
    rep = level_report.report(fx, dcc=rec)
    assert rep["dcc_alpha_flips"] == 0 and rep["dcc_p_abs_err_max"] == 0.0 and rep["dcc_stat_rel_err_max"] == 0.0


@pytest.mark.slow
def test_polished_point_is_stationary_in_extended_precision():
    """Fit 4580 of the 500x50 level batch (|S| = 4, two smooths near
    lambda = e^23 and e^25): the polished log(lambda) has a relative GCV
    gradient below 1e-13 when V is evaluated in 30-digit arithmetic (a
    polish on the SVD route's derivatives stopped where it was 1e-12)."""
    mp = pytest.importorskip("mpmath")
    from threadpoolctl import threadpool_limits
    from fastkpc_b200 import workloads
    from tests.golden import level_report
    fx = level_report.load()
    X, _ = workloads.level_batch_500x50(count=len(fx["x"]))
    i = 4580
    t = int(fx["fit_target"][i])
    S = [int(v) for v in fx["fit_S"][i] if v >= 0]
    d = tprs.design(X, S)
    with threadpool_limits(limits=1):
        _, info = gcv.fit(gcv.Prepared(d), X[:, t])
    assert np.max(np.abs(info["log_sp"] - fx["fit_log_sp"][i][:len(S)])) < 1e-10
    mp.mp.dps = 30
    n, q = d["X"].shape
    Xm = mp.matrix(d["X"].tolist())
    XtX = Xm.T * Xm
    ym = mp.matrix(X[:, t].tolist())
    Xty = Xm.T * ym
    yy = (ym.T * ym)[0]
    blocks = [(mp.matrix(b.tolist()), off) for b, off in zip(d["blocks"], d["offsets"])]

    def V(rho):
        A = XtX.copy()
        for (b, off), r in zip(blocks, rho):
            lam = mp.exp(r)
            for a in range(b.rows):
                for c in range(b.cols):
                    A[off + a, off + c] += lam * b[a, c]
        Ai = mp.inverse(A)
        beta = Ai * Xty
        rss = yy - 2 * (Xty.T * beta)[0] + (beta.T * XtX * beta)[0]
        edf = sum((Ai * XtX)[k, k] for k in range(q))
        return n * rss / (n - edf) ** 2

    rho = [mp.mpf(float(v)) for v in info["log_sp"]]
    h = mp.mpf("1e-8")
    v0 = V(rho)
    for j in (0, 3):  # the two well-determined coordinates
        rp, rm = list(rho), list(rho)
        rp[j] += h
        rm[j] -= h
        assert abs((V(rp) - V(rm)) / (2 * h) / v0) < 1e-13


def test_skeleton_fixture_is_the_oracle():
    """The committed 351x48 (seed 537) oracle skeletons: the trace holds
    n.edgetests rows, deletions match the adjacency, and the oracle re-run on
    the first level-1 tests reproduces their p-values."""
    from threadpoolctl import threadpool_limits
    from fastkpc_b200 import workloads
    with np.load(golden_path("skeleton351x48_s537_oracle.npz")) as f:
        fx = {k: f[k] for k in f.files}
    X = workloads.skeleton_351x48(int(fx["seed"]))
    cache = skeleton.ResidualCache(X)
    for method in ("hsic.gamma", "dcc.gamma"):
        key = method.replace(".", "_") + "_"
        assert len(fx[key + "trace_p"]) == int(fx[key + "n_edgetests"].sum())
        deleted = int(fx[key + "trace_deletes"].sum())
        edges = int(fx[key + "adjacency"].sum()) // 2
        assert edges + deleted == 48 * 47 // 2
        rows = np.nonzero(fx[key + "trace_level"] == 1)[0][:6]
        with threadpool_limits(limits=1):
            for k in rows:
                S = [int(v) for v in fx[key + "trace_S"][k] if v >= 0]
                pv = skeleton.ci_pvalue(cache, method, int(fx[key + "trace_x"][k]), int(fx[key + "trace_y"][k]), S)
                assert abs(pv - fx[key + "trace_p"][k]) <= 1e-12
