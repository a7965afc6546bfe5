"""The device thin-plate eigensolvers against the oracle's dense
eigen-decomposition (B200).

A bivariate smooth (m = 2, k = 30) needs the 30 eigenpairs of largest
magnitude of its eta matrix over the unique locations
(fastkpc/src/full_cuda_ci_native_setup.cpp:114-152, 303).  The device takes a
design to the block Lanczos when 120 <= n_u <= 512 and to the single-vector
Lanczos otherwise; the oracle takes numpy's dense symmetric solver on the
same matrix.  Bars: Ritz values within 1e-12 of max |value|; Ritz vectors
(unit norm, largest-magnitude entry positive, the same unique-location
order) within 1e-10 entrywise -- an eigenvector moves by its residual over
the gap to the next eigenvalue, and the measured maxima are printed.
"""
import json

import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from oracle import tprs
from tests.conftest import golden_path

pytestmark = pytest.mark.gpu

VAL_TOL = 1e-12
VEC_TOL = 1e-10


def oracle_pairs(X, a, b):
    cols = X[:, [min(a, b), max(a, b)]]
    shifts = np.array([tprs.r_mean(cols[:, j]) for j in range(2)])
    uniq, _ = tprs.sorted_unique(cols - shifts)
    diff = uniq[:, None, :] - uniq[None, :, :]
    E = tprs.eta_of_r2(2, 2, np.sum(diff * diff, axis=2), tprs.eta_constant(2, 2))
    return tprs.top_magnitude_eigen(E, 30)


def _ten_levels(n=300, seed=13):
    rs = np.random.default_rng(seed)
    X = rs.normal(size=(n, 6))
    lv = np.array([0.0, 1.1, 2.5, 3.2, 4.8, 6.0, 7.7, 9.1, 10.4, 12.9])
    X[:, 0] = lv[rs.integers(0, 10, size=n)]
    X[:, 1] = lv[rs.integers(0, 10, size=n)] * 0.7 + 0.13
    return np.asfortranarray(X)


def _twelve_levels(n=300, seed=1):
    """Two columns of 12 jittered levels: 127 unique locations, the block
    path's smallest range (leading dimension 128: four of the eight warps own
    a row block)."""
    rs = np.random.default_rng(seed)
    lv = np.linspace(0.0, 11.0, 12) + rs.normal(scale=0.05, size=12)
    X = np.empty((n, 3))
    X[:, 0] = lv[rs.integers(0, 12, size=n)]
    X[:, 1] = lv[rs.integers(0, 12, size=n)] * 0.9 + 0.2
    X[:, 2] = rs.normal(size=n)
    return np.asfortranarray(X)


def cases():
    dev = np.load(golden_path("dev500x50.npz"))["data"]
    sem351 = workloads.skeleton_351x48(537)
    sem1000 = workloads.nonlinear_sem(1000, 12, 0.3, 31)[0]
    return [("dev500", dev, 0, 1, "block"), ("dev500", dev, 17, 42, "block"), ("dev500", dev, 5, 49, "block"),
            ("sem351x48", sem351, 3, 40, "block"), ("sem1000x12", sem1000, 3, 7, "single"),
            ("ten_levels", _ten_levels(), 0, 1, "single"), ("twelve_levels", _twelve_levels(), 0, 1, "block")]


@pytest.mark.parametrize("case", range(7))
def test_device_ritz_pairs_match_dense_eigen(lib_built, case):
    name, X, a, b, path = cases()[case]
    got = fk.tprs_export(X, a, b)
    assert got["path"] == path and got["ok"]
    vals, vecs = oracle_pairs(X, a, b)
    assert got["n_u"] == vecs.shape[0]
    scale = np.max(np.abs(vals))
    verr = float(np.max(np.abs(got["values"] - vals)) / scale)
    uerr = float(np.max(np.abs(got["vectors"] - vecs)))
    print(json.dumps({"case": name, "columns": [a, b], "path": path, "n_u": got["n_u"],
                      "value_rel_err": verr, "vector_abs_err": uerr}))
    assert verr <= VAL_TOL
    assert uerr <= VEC_TOL


def test_design_outside_the_device_range_is_not_taken(lib_built):
    """Fewer unique locations than the single-vector step count: the host
    builds that smooth, and the export says so."""
    rs = np.random.default_rng(3)
    X = np.asfortranarray(np.column_stack([rs.integers(0, 7, size=200).astype(float),
                                           rs.integers(0, 7, size=200).astype(float), rs.normal(size=200)]))
    got = fk.tprs_export(X, 0, 1)
    assert got["path"] is None and got["n_u"] <= 49
