"""Rank-deficient designs: magic's rank rule on the device (B200).

A conditioning set that holds the same variable twice (column 49 of the
reference's 500 x 50 development dataset overwritten by column 7) gives an
additive design whose augmented system [R; sqrt(lambda) root'] has a null
direction: the two smooths' linear terms coincide and no penalty sees them.
mgcv's magic, the reference (rank_tolerance = sqrt(eps),
fastkpc/src/cuda/mgcv_multi_penalty_gcv.hpp:230) and the oracle's truncated
SVD drop singular values below sqrt(eps) times the largest; the fits drop
the coefficient of the negligible pivot instead, which leaves the same fitted
values.  Bars: residuals within 1e-9 of the oracle's (relative to max |r|),
p-values within 1e-9, and every such test flagged FKPC_FLAG_RANK_TRUNCATED.
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from oracle import gcv, skeleton, tprs

pytestmark = pytest.mark.gpu

FITS = [(0, [7, 12, 49]), (3, [5, 7, 20, 49]), (10, [7, 11, 13, 17, 49]),
        (1, [2, 7, 9, 14, 21, 30, 33, 38, 41, 44, 46, 48, 49])]


@pytest.fixture(scope="module")
def dup(dev500):
    d = dev500["data"].copy()
    d[:, 49] = d[:, 7]
    return np.asfortranarray(d)


def test_duplicated_variable_fits_match_truncated_oracle(lib_built, dup):
    resid, lsp, status = fk.regress_batch(dup, FITS)
    assert (status == 0).all(), status
    errs = []
    for k, (t, S) in enumerate(FITS):
        prep = gcv.Prepared(tprs.design(dup, S))
        r, info = gcv.fit(prep, dup[:, t])
        errs.append(float(np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))))
    print(json.dumps({"sizes": [len(S) for _, S in FITS], "residual_rel_err": errs}))
    assert max(errs) <= 1e-9


@pytest.mark.parametrize("method", ["dcc.gamma", "hsic.gamma"])
def test_duplicated_variable_tests_are_flagged_and_match(lib_built, dup, method):
    tests = [(0, 30, [7, 12, 49]), (3, 40, [5, 7, 20, 49]), (6, 8, [1, 2, 3])]
    rec, _ = fk.ci_level_batch(dup, tests, ci_method=method)
    cache = skeleton.ResidualCache(dup)
    perr = max(abs(rec["p_value"][k] - skeleton.ci_pvalue(cache, method, *t)) for k, t in enumerate(tests))
    flags = [int(f) for f in rec["flags"]]
    print(json.dumps({"method": method, "p_abs_err_max": perr, "flags": flags}))
    assert perr <= 1e-9
    assert all(f & fk.FLAG_RANK_TRUNCATED for f in flags[:2])
    assert not flags[2] & fk.FLAG_RANK_TRUNCATED
