"""The C ABI library: loads, exports every declared symbol, host-only set-up.

No compute runs here (no GPU in the CPU suite); the design set-up is host
code and is checked against the oracle's mgcv thin-plate restatement.
"""
import os
import re

import numpy as np
import pytest

import fastkpc_b200 as fk
from oracle import gcv, tprs
from tests.conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names.update(re.findall(r"FKPC_API\s+[\w\s\*]+?\b(fkpc_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol(lib_built):
    names = declared_symbols()
    assert {"fkpc_skeleton_run", "fkpc_ci_level_batch", "fkpc_ci_plain_one", "fkpc_gcv_adjoint",
            "fkpc_last_error", "fkpc_result_free"} <= names
    for name in names:
        assert hasattr(lib_built, name), name


def test_abi_version_and_defaults(lib_built):
    assert lib_built.fkpc_abi_version() == 5
    o = fk.make_options()
    assert o.alpha == 0.1 and o.num_col == 35 and o.index == 1.0 and o.strict == 1
    assert o.selection == 0 and fk.make_options(selection="gn_newton").selection == 1
    with pytest.raises(ValueError):
        fk.make_options(selection="bfgs")


def test_envelope_errors_are_raised_before_any_device_work(lib_built):
    d = np.random.default_rng(0).normal(size=(50, 4))
    with pytest.raises(fk.FkpcError) as e:
        fk.ci_level_batch(d, [(0, 1, [])], alpha=0.2)
    assert e.value.status == 1 and "alpha" in str(e.value)
    with pytest.raises(fk.FkpcError):
        fk.ci_level_batch(d, [(0, 1, [])], ci_method="hsic.perm")  # no seed
    with pytest.raises(ValueError):
        fk.fastkpc_compatible_cuda_skeleton(d, 0.1, options={"bogus": 1})


@pytest.mark.parametrize("S", [[3], [3, 7], [1, 5, 9], [2, 11, 17, 40]])
def test_host_design_matches_oracle(lib_built, dev500, S):
    d = dev500["data"]
    cd = fk.design_export(d, S)
    od = tprs.design(d, S)
    assert cd["q"] == od["X"].shape[1]
    assert np.max(np.abs(cd["X"] - od["X"])) < 1e-9
    assert np.allclose(cd["initial_log_sp"], np.log(od["initial_sp"]), rtol=0, atol=1e-12)
    # the GCV fit on the library's design equals the fit on the oracle design
    blocks = [cd["penalties"][j][o:o + b.shape[0], o:o + b.shape[0]]
              for j, (o, b) in enumerate(zip(od["offsets"], od["blocks"]))]
    desc = {"X": cd["X"], "blocks": blocks, "offsets": od["offsets"], "ranks": od["ranks"],
            "initial_sp": np.exp(cd["initial_log_sp"])}
    rc, ic = gcv.fit(gcv.Prepared(desc), d[:, 20])
    ro, io = gcv.fit(gcv.Prepared(od), d[:, 20])
    assert np.max(np.abs(rc - ro)) <= 1e-10 * np.max(np.abs(ro))


def test_host_lanczos_restarts_on_near_duplicate_locations(lib_built):
    """Column 43 of the n=351, p=48 SEM with seed 619: 320 of its 351 values
    lie within 1e-9 of each other, so the eta matrix of its smooth is
    numerically rank deficient and Lanczos meets an invariant subspace before
    it has k = 10 Ritz pairs.  The set-up restarts from a new orthogonal start
    vector instead of failing (the near-null pairs it adds are rounding-level,
    as any dense eigensolver's would be)."""
    from fastkpc_b200 import workloads
    X = workloads.skeleton_351x48(619)
    c = np.sort(X[:, 43])
    assert np.sum(np.diff(c) < 1e-9) > 300
    d = fk.design_export(X, [43])
    assert d["q"] == 10 and np.all(np.isfinite(d["X"]))
    d2 = fk.design_export(X, [43, 7])
    assert d2["q"] == 30 and np.all(np.isfinite(d2["X"]))


@pytest.mark.parametrize("method", ["dcc.perm", "hsic.perm"])
def test_permutation_tables_are_the_oracle_stream(lib_built, method):
    """The library's R stream draws the oracle's tables test after test
    (fastkpc/src/full_cuda_ci_one_call.cpp:464-567), including sizes whose
    R_unif_index bit count changes (n = 2, 33, 64, 65)."""
    from oracle import rng
    draw = rng.dcc_permutations if method == "dcc.perm" else rng.hsic_permutations
    for seed, n, reps, count in [(537, 37, 19, 5), (1, 2, 4, 3), (2024, 33, 7, 2), (9, 64, 3, 2), (9, 65, 3, 2)]:
        got = fk.permutation_tables(seed, method, n, reps, count)
        s = rng.RStream(seed)
        want = np.array([draw(s, n, reps) for _ in range(count)])
        assert np.array_equal(got, want), (seed, n)
    with pytest.raises(fk.FkpcError):
        fk.permutation_tables(1, "dcc.gamma", 10, 2, 1)
    with pytest.raises(fk.FkpcError):
        fk.permutation_tables(1, method, 1, 2, 1)
