"""Conditioning sets with |S| > 12: the wide fit class (q <= 560, |S| <= 62,
working set in global memory) against the oracle (B200).

The reference's envelope is p <= 64 with m.max = p - 2, so a default-Inf
skeleton can reach |S| = 62 (fastkpc/src/full_cuda_ci_one_call.cpp:5052-5060;
capacity q <= 559, m <= 62 in fastkpc/src/cuda/mgcv_multi_penalty_gcv.hpp:28-29).
Data: the reference's 500 x 50 development dataset.  Bars: residuals within
1e-10 of the oracle's (relative to max |r|), CI p-values within 1e-9, plain
and batched forms bit-identical.
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from oracle import gcv, skeleton, tprs

pytestmark = pytest.mark.gpu

RESID_TOL = 1e-10
WIDE_FITS = [(0, [1, 3, 5, 7, 9, 11, 13, 19, 21, 23, 25, 27, 29]),
             (2, list(range(10, 26))),
             (4, list(range(5, 25))),
             (49, [2 * i + 1 for i in range(24)])]


def test_wide_residuals_match_oracle(lib_built, dev500):
    d = dev500["data"]
    fits = WIDE_FITS + [(8, [0, 12, 24, 36, 48])]  # one narrow fit in the same batch
    resid, lsp, status = fk.regress_batch(d, fits)
    assert (status == 0).all(), status
    errs = []
    for k, (t, S) in enumerate(fits):
        prep = gcv.Prepared(tprs.design(d, S))
        r, info = gcv.fit(prep, d[:, t])
        err = float(np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r)))
        errs.append(err)
        assert err <= RESID_TOL, (t, len(S), err)
        assert np.all(np.isnan(lsp[k, len(S):]))
    print(json.dumps({"sizes": [len(S) for _, S in fits], "residual_rel_err": errs}))


@pytest.mark.parametrize("method", ["dcc.gamma", "hsic.gamma"])
def test_wide_ci_tests_match_oracle(lib_built, dev500, method):
    d = dev500["data"]
    tests = [(0, 30, [1, 3, 5, 7, 9, 11, 13, 19, 21, 23, 25, 27, 29]),
             (2, 40, list(range(10, 26))),
             (44, 45, list(range(0, 13))),
             (6, 7, [0, 1, 2])]
    rec, stats = fk.ci_level_batch(d, tests, ci_method=method)
    cache = skeleton.ResidualCache(d)
    perr = 0.0
    for k, t in enumerate(tests):
        want = skeleton.ci_pvalue(cache, method, t[0], t[1], t[2])
        perr = max(perr, abs(rec["p_value"][k] - want))
    print(json.dumps({"method": method, "p_abs_err_max": perr, "device_ms": stats["device_ms"]}))
    assert perr <= 1e-9
    plain, _ = fk.ci_level_batch(d, tests, ci_method=method, mode="plain")
    for key in ("p_value", "statistic"):
        assert np.array_equal(plain[key], rec[key]), key


def test_design_wider_than_the_data_is_rejected(lib_built, dev500):
    d = dev500["data"][:100]
    with pytest.raises(fk.FkpcError, match="width must be below n"):
        fk.regress_batch(d, [(0, list(range(1, 13)))])  # q = 109 >= n = 100
