"""All 4096 triples of the 500 x 50 level batch against the oracle (B200).

The oracle's records and residual summaries come from the committed fixture
``tests/golden/level500x50_oracle.npz`` (``make_level_fixture.py``).  Every
call goes through the C ABI.  Bars (the tolerances of the CI path):

* residuals within 1e-10 relative (max-abs error over max |r|) on the 301
  fits stored in full; on all 6005 fits |(r - r_o) . z| <= 1e-10 |r_o| |z|
  for four fixed vectors z (what a 1e-10 relative error allows) and |r|^2
  within 2e-10 relative; selected log(lambda) within 1e-8 where the GCV
  score's curvature decides it (entries below 15), the rest being smooths
  pushed towards lambda = infinity, where V is flat and the residual does not
  move;
* statistics, means and variances within 1e-10 relative;
* gamma p (dcc.gamma exact screen, hsic.gamma) within 1e-12 absolute on every
  triple whose two fits select the oracle's log(lambda) to 1e-11 (4058 of
  4096); within 1e-11 on the rest.  There mgcv magic's stopping rule fired
  outside the Newton region (|grad V| / V up to 3e-4, where the terminal
  polish does not apply), and two implementations of the same search, whose
  Newton steps round differently, end up to 1e-9 apart in log(lambda): a
  property of the reference's loose stopping rule, not of either side;
* guard-band (low-rank) p within 1e-10 (its 35 eigenpairs come from Lanczos
  on the device and a dense eigensolver in the oracle);
* no alpha-boundary flip and no guard-band routing flip.

The measured errors are printed (``pytest -s``) as one JSON line per test.
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from tests.golden import level_report

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fx():
    return level_report.load()


@pytest.fixture(scope="module")
def data(fx):
    X, triples = workloads.level_batch_500x50(count=len(fx["x"]))
    assert triples == level_report.triples(fx), "fixture and workload generator disagree"
    return X


@pytest.fixture(scope="module")
def fitted(lib_built, fx, data):
    resid, lsp, status = fk.regress_batch(data, level_report.fits(fx), max_penalties=4)
    assert np.all(status == 0)
    return resid, lsp


def test_level_fits_match_oracle(fx, fitted):
    resid, lsp = fitted
    rep = level_report.report(fx, residuals=resid, log_sp=lsp)
    print(json.dumps({"stage": "fit", **rep}))
    assert rep["residual_rel_err_max"] <= 1e-10
    assert rep["residual_projection_bound_max"] <= 1e-10
    assert rep["residual_norm2_rel_err_max"] <= 2e-10
    assert rep["log_sp_abs_err_max_below_15"] <= 1e-8


def test_level_dcc_gamma_matches_oracle(fx, data, fitted):
    rec, _ = fk.ci_level_batch(data, level_report.triples(fx), ci_method="dcc.gamma")
    assert np.all(rec["status"] == 0)
    rep = level_report.report(fx, dcc=rec, log_sp=fitted[1])
    print(json.dumps({"stage": "dcc.gamma", **rep}))
    assert rep["dcc_guard_route_flips"] == 0
    assert rep["dcc_alpha_flips"] == 0
    assert rep["dcc_stat_rel_err_max"] <= 1e-10
    assert rep["dcc_moment_rel_err_max"] <= 1e-10
    assert rep["triples_fits_agreeing"] >= 4000
    assert rep["dcc_p_exact_abs_err_max_agreeing"] <= 1e-12
    assert rep["dcc_p_exact_abs_err_max"] <= 1e-11
    assert rep["dcc_p_lowrank_abs_err_max"] <= 1e-10


def test_level_hsic_gamma_matches_oracle(fx, data, fitted):
    rec, _ = fk.ci_level_batch(data, level_report.triples(fx), ci_method="hsic.gamma")
    assert np.all(rec["status"] == 0)
    rep = level_report.report(fx, hsic=rec, log_sp=fitted[1])
    print(json.dumps({"stage": "hsic.gamma", **rep}))
    assert rep["hsic_alpha_flips"] == 0
    assert rep["hsic_stat_rel_err_max"] <= 1e-10
    assert rep["hsic_moment_rel_err_max"] <= 1e-10
    assert rep["triples_fits_agreeing"] >= 4000
    assert rep["hsic_p_abs_err_max_agreeing"] <= 1e-12
    assert rep["hsic_p_abs_err_max"] <= 1e-11
