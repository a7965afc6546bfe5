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
