"""CUDA path against the oracle and the reference fixtures (needs a B200).

Every call goes through the C ABI (libfastkpc_b200.so).  Tolerances:
statistics and gamma p-values within 1e-12 of the oracle (scipy gamma tail),
residuals within 1e-10 relative to their maximum, permutation p-values and
all graph / sepset / decision / test-count outcomes exact.
"""
import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import workloads
from oracle import gcv, rng, skeleton, stats, tprs

pytestmark = pytest.mark.gpu

STAT_TOL = 1e-12
RESID_TOL = 1e-10


@pytest.fixture(scope="module")
def lib(lib_built):
    return lib_built


def _residual_pool(n, m, seed):
    rs = np.random.default_rng(seed)
    base = rs.normal(size=(n, m))
    # dependent columns so p-values spread over (0, 1)
    base[:, 1] = np.tanh(base[:, 0]) + 0.7 * base[:, 1]
    base[:, 3] = np.sin(2 * base[:, 2]) * 0.5 + base[:, 3]
    base[:, 5] = 0.2 * base[:, 4] ** 2 + base[:, 5]
    return np.asfortranarray(base)


@pytest.mark.parametrize("n", [60, 200, 500])
def test_dcov_exact_statistics_match_oracle(lib, n):
    R = _residual_pool(n, 8, n)
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 7), (1, 6)]
    rec = fk.stat_batch(R, pairs, ci_method="dcc.gamma")
    for k, (a, b) in enumerate(pairs):
        o = stats.dcov_gamma_exact(R[:, a], R[:, b])
        assert abs(rec["p_exact"][k] - o["p_value"]) <= STAT_TOL
        if rec["flags"][k] & fk.FLAG_GUARDED:
            # guard band: the record carries the low-rank (legacy) statistic
            assert 0.05 <= o["p_value"] <= 0.15
            o = stats.dcov_gamma_legacy(R[:, a], R[:, b], 35)
            assert abs(rec["p_value"][k] - o["p_value"]) <= 1e-10
            assert rec["statistic"][k] == pytest.approx(o["statistic"], rel=1e-10)
            continue
        assert rec["statistic"][k] == pytest.approx(o["statistic"], rel=STAT_TOL)
        assert rec["mean"][k] == pytest.approx(o["mean"], rel=STAT_TOL)
        assert rec["variance"][k] == pytest.approx(o["variance"], rel=STAT_TOL)
        assert abs(rec["p_value"][k] - o["p_value"]) <= STAT_TOL


def test_dcov_guard_band_uses_low_rank_refinement(lib):
    import json
    from tests.conftest import golden_path
    cases = json.load(open(golden_path("legacy_dcov_gamma.json")))["cases"]
    R = np.asfortranarray(np.column_stack([np.array(c[k]) for c in cases for k in ("rx", "ry")]))
    pairs = [(2 * i, 2 * i + 1) for i in range(len(cases))]
    rec = fk.stat_batch(R, pairs, ci_method="dcc.gamma")
    for k, c in enumerate(cases):
        ex = stats.dcov_gamma_exact(np.array(c["rx"]), np.array(c["ry"]))
        guarded = 0.05 <= ex["p_value"] <= 0.15
        assert bool(rec["flags"][k] & fk.FLAG_GUARDED) == guarded, c["case_id"]
        if guarded:
            # reference legacy values (RSpectra-based, 1e-8) and the dense-eigen oracle
            assert abs(rec["p_value"][k] - c["p_value"]) <= 1e-8, c["case_id"]
            lg = stats.dcov_gamma_legacy(np.array(c["rx"]), np.array(c["ry"]), 35)
            assert abs(rec["p_value"][k] - lg["p_value"]) <= 1e-10, c["case_id"]
            assert (rec["p_value"][k] >= 0.1) == c["delete_edge"], c["case_id"]


@pytest.mark.parametrize("n", [60, 200, 500])
def test_hsic_gamma_matches_oracle(lib, n):
    R = _residual_pool(n, 8, 7 + n)
    pairs = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 7)]
    rec = fk.stat_batch(R, pairs, ci_method="hsic.gamma")
    for k, (a, b) in enumerate(pairs):
        o = stats.hsic_gamma(R[:, a], R[:, b], 1.0, 35)
        assert rec["statistic"][k] == pytest.approx(o["statistic"], rel=1e-11)
        assert rec["mean"][k] == pytest.approx(o["mean"], rel=1e-11)
        assert rec["variance"][k] == pytest.approx(o["variance"], rel=1e-10)
        assert abs(rec["p_value"][k] - o["p_value"]) <= 1e-11


@pytest.mark.parametrize("method", ["dcc.perm", "hsic.perm"])
def test_permutation_statistics_match_oracle(lib, method):
    n, R_ = 80, 40
    R = _residual_pool(n, 6, 11)
    pairs = [(0, 1), (2, 3), (4, 5)]
    stream = rng.RStream(2024)
    gen = rng.dcc_permutations if method == "dcc.perm" else rng.hsic_permutations
    perms = np.stack([gen(stream, n, R_) for _ in pairs])
    rec = fk.stat_batch(R, pairs, ci_method=method, permutations=perms, seed=1, replicates=R_)
    for k, (a, b) in enumerate(pairs):
        if method == "dcc.perm":
            o = stats.dcc_perm(R[:, a], R[:, b], perms[k])
        else:
            o = stats.hsic_perm(R[:, a], R[:, b], perms[k], 1.0, 35)
        assert rec["p_value"][k] == o["p_value"]
        assert rec["statistic"][k] == pytest.approx(o["statistic"], rel=1e-11)


FITS = [(0, [3]), (20, [3]), (7, [2, 11]), (30, [5, 6]), (20, [1, 5, 9]), (0, [1, 5, 9]),
        (41, [2, 11, 17, 40]), (8, [0, 12, 24, 36, 48]), (15, [1, 3, 5, 7, 9, 11, 13, 19])]


def test_regress_residuals_match_oracle(lib, dev500):
    d = dev500["data"]
    resid, lsp, status = fk.regress_batch(d, FITS)
    assert (status == 0).all()
    for k, (t, S) in enumerate(FITS):
        prep = gcv.Prepared(tprs.design(d, S))
        r, info = gcv.fit(prep, d[:, t])
        err = np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))
        assert err <= RESID_TOL, (t, S, err)
        assert np.allclose(lsp[k, :len(S) if len(S) > 2 else 1], info["log_sp"], atol=1e-5)


def _oracle_p(cache, t, method="dcc.gamma"):
    return skeleton.ci_pvalue(cache, method, t[0], t[1], t[2])


def test_level_batch_matches_oracle_and_plain(lib):
    X, triples = workloads.level_batch_500x50(count=48)
    rec, st = fk.ci_level_batch(X, triples)
    assert st["pairs"] == 48 and st["kernel_launches"] > 0
    cache = skeleton.ResidualCache(X)
    for k, t in enumerate(triples):
        p = _oracle_p(cache, t)
        assert abs(rec["p_value"][k] - p) <= 1e-9, (t, rec["p_value"][k], p)
        assert (rec["p_value"][k] >= 0.1) == (p >= 0.1)
    plain = [fk.ci_plain_one(X, t[0], t[1], t[2]) for t in triples[:12]]
    for k, r in enumerate(plain):
        assert r["p_value"] == rec["p_value"][k]


def test_hsic_level_batch_matches_oracle(lib):
    X, triples = workloads.level_batch_500x50(count=24)
    rec, _ = fk.ci_level_batch(X, triples, ci_method="hsic.gamma")
    cache = skeleton.ResidualCache(X)
    for k, t in enumerate(triples):
        p = _oracle_p(cache, t, "hsic.gamma")
        assert abs(rec["p_value"][k] - p) <= 1e-9, (t, rec["p_value"][k], p)


def test_skeleton_500x50_matches_reference_fixture(lib, dev500, dev500_trace):
    out = fk.fastkpc_compatible_cuda_skeleton(dev500["data"], 0.1, options={"trace_level": "logical", "numCol": 35})
    assert out["n_edgetests"] == dev500["n_edgetests"].tolist()
    assert np.array_equal(out["adjacency"].astype(np.int8), dev500["adjacency"])
    tasks = out["tasks"]
    ref = {(r["level"], r["x"], r["y"], tuple(r["S"])): r for r in dev500_trace["logical_trace"]}
    assert len(tasks["level"]) == len(ref)
    for k in range(len(tasks["level"])):
        key = (int(tasks["level"][k]), int(tasks["x"][k]), int(tasks["y"][k]), tuple(tasks["S"][k]))
        assert bool(tasks["native_edge_deleted"][k]) == ref[key]["deletes_edge"], key
    ref_sep = {(i, j): s for i, j, s in dev500_trace["sepsets"]}
    for (i, j), s in ref_sep.items():
        assert sorted(out["sepsets"][i][j]) == s


@pytest.mark.parametrize("method", ["hsic.gamma", "dcc.gamma"])
def test_skeleton_200x10_matches_oracle(lib, method):
    X = workloads.skeleton_200x10()
    out = fk.fastkpc_compatible_cuda_skeleton(X, 0.1, options={"ci_method": method, "numCol": 35,
                                                               "trace_level": "logical"})
    ora = skeleton.skeleton(X, 0.1, method)
    assert out["n_edgetests"] == ora["n_edgetests"].tolist()
    assert np.array_equal(out["adjacency"], ora["adjacency"])
    for k, row in enumerate(ora["trace"]):
        assert abs(out["tasks"]["p_used"][k] - row["p_value"]) <= 1e-9


@pytest.mark.parametrize("method", ["dcc.perm", "hsic.perm"])
def test_permutation_skeleton_matches_oracle_stream(lib, method):
    X = workloads.nonlinear_sem(60, 5, 0.4, 9)[0]
    opts = {"ci_method": method, "numCol": 35, "trace_level": "logical",
            "permutation_params": {"replicates": 30, "seed": 42, "include_observed": True}}
    out = fk.fastkpc_compatible_cuda_skeleton(X, 0.1, options=opts)
    ora = skeleton.skeleton(X, 0.1, method, replicates=30, seed=42)
    assert out["n_edgetests"] == ora["n_edgetests"].tolist()
    assert np.array_equal(out["adjacency"], ora["adjacency"])
    got = sorted(zip(out["tasks"]["level"], out["tasks"]["x"], out["tasks"]["y"],
                     map(tuple, out["tasks"]["S"]), out["tasks"]["p_used"]))
    exp = sorted((r["level"], r["x"], r["y"], tuple(r["S"]), r["p_value"]) for r in ora["trace"])
    assert [g[:4] for g in got] == [e[:4] for e in exp]
    assert [g[4] for g in got] == [e[4] for e in exp]


def test_wide_additive_fits_match_oracle(lib):
    """|S| = 9, 10, 12 (q = 82, 91, 109): the widest fit class, whose working
    set lives in global memory, against the oracle at the residual tolerance."""
    X, _ = workloads.uneven_batch_500x64(count=8)
    fits = [(0, [3, 7, 11, 15, 19, 23, 27, 31, 35]), (5, [1, 2, 8, 13, 21, 34, 40, 44, 50, 55]),
            (9, [2, 4, 6, 10, 12, 16, 18, 22, 26, 30, 38, 62])]
    resid, lsp, status = fk.regress_batch(X, fits)
    assert (status == 0).all()
    for k, (t, S) in enumerate(fits):
        prep = gcv.Prepared(tprs.design(X, S))
        r, info = gcv.fit(prep, X[:, t])
        err = np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))
        assert err <= RESID_TOL, (t, len(S), err)
    t, S = fits[1]
    prep = gcv.Prepared(tprs.design(X, S))
    rho = np.log(prep.initial_sp)
    a = fk.gcv_adjoint(X, t, S, rho[None, :])
    V, g, H = gcv.gcv_value_grad_hess(prep, X[:, t], rho)
    assert abs(a["score"][0] - V) <= 1e-10 * V
    assert np.max(np.abs(a["grad"][0] - g)) <= 1e-8 * np.max(np.abs(g))
    assert np.max(np.abs(a["hessian"][0] - H)) <= 1e-8 * np.max(np.abs(H))


def _uneven_triples(X, count, seed):
    """Triples of the n=500, p=64 batch with a spread of |S| up to 12."""
    rs = np.random.default_rng(seed)
    p = X.shape[1]
    out = []
    for k in (0, 1, 2, 3, 4, 6, 9):
        cols = rs.choice(p, size=k + 2, replace=False)
        out.append((int(cols[0]), int(cols[1]), sorted(int(c) for c in cols[2:])))
    return out[:count]


@pytest.mark.parametrize("method", ["dcc.perm", "hsic.perm"])
def test_uneven_permutation_batch_matches_oracle_stream(lib, method):
    """Uneven widths (|S| up to 9 here) with permutation nulls: the level
    batch consumes the seeded R stream test by test; p-values exact."""
    X, _ = workloads.uneven_batch_500x64(count=8)
    triples = _uneven_triples(X, 7, 11)
    R_ = 40
    rec, _ = fk.ci_level_batch(X, triples, ci_method=method, seed=7, replicates=R_)
    stream = rng.RStream(7)
    gen = rng.dcc_permutations if method == "dcc.perm" else rng.hsic_permutations
    cache = skeleton.ResidualCache(X)
    for k, (x, y, S) in enumerate(triples):
        perms = gen(stream, X.shape[0], R_)
        assert rec["p_value"][k] == skeleton.ci_pvalue(cache, method, x, y, S, perms=perms), (x, y, S)


def test_permutation_batch_chunks_keep_the_stream_order(lib):
    """600 tests with R = 1000 exceed one permutation-table chunk (about
    1 GiB, 536 tests at n = 500): the chunked batch equals the plain per-test
    form, which consumes the same stream one test at a time."""
    X, triples = workloads.uneven_batch_500x64(count=800)
    triples = [t for t in triples if len(t[2]) <= 3][:600]
    assert len(triples) == 600
    kw = dict(ci_method="dcc.perm", seed=3, replicates=1000)
    batched, _ = fk.ci_level_batch(X, triples, **kw)
    plain, _ = fk.ci_level_batch(X, triples, mode="plain", **kw)
    assert np.array_equal(batched["p_value"], plain["p_value"])
    assert np.array_equal(batched["statistic"], plain["statistic"])


def test_sharded_skeleton_single_rank_equals_direct(lib):
    """The multi-GPU driver (level evaluator hook, records gathered per level)
    run as a one-rank group on this GPU gives the direct skeleton exactly."""
    import os
    import socket

    import torch.distributed as dist

    from fastkpc_b200 import distributed
    X = workloads.skeleton_200x10()
    opts = {"numCol": 35, "trace_level": "logical"}
    direct = fk.fastkpc_compatible_cuda_skeleton(X, 0.1, options=opts)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        _, _, o, _ = fk._skeleton_setup(X, 0.1, None, opts)
        inner = distributed.level_batch_evaluator(X, o)
        seen = []

        def evaluate(tests):
            seen.extend(tuple(t[2]) for t in tests)
            return inner(tests)
        sharded = distributed.sharded_skeleton(X, 0.1, options=opts, evaluate=evaluate)
        # the rank's session keeps its caches across levels: every design and
        # every per-variable smooth is set up once, however many levels use it
        sets = {S for S in seen if S}
        smooth_vars = {v for S in sets if len(S) != 2 for v in S}
        assert sum(st["designs_built"] for st in inner.stats) == len(sets)
        assert sum(st["smooths_built"] for st in inner.stats) == len(smooth_vars)
        assert sum(st["smooths_built"] > 0 for st in inner.stats) >= 1
    finally:
        dist.destroy_process_group()
    assert np.array_equal(sharded["adjacency"], direct["adjacency"])
    assert np.array_equal(sharded["pMax"], direct["pMax"])
    assert sharded["sepsets"] == direct["sepsets"]
    assert sharded["n_edgetests"] == direct["n_edgetests"]


def test_bivariate_designs_set_up_on_the_device_match_oracle(lib, dev500):
    """40 new |S| = 2 designs in one call, set up with the device thin-plate
    Lanczos: residuals against the oracle at the tolerance."""
    d = dev500["data"]
    rs = np.random.default_rng(5)
    fits = []
    seen = set()
    while len(fits) < 40:
        a, b, t = (int(v) for v in rs.choice(d.shape[1], size=3, replace=False))
        S = tuple(sorted((a, b)))
        if S in seen:
            continue
        seen.add(S)
        fits.append((t, list(S)))
    resid, lsp, status = fk.regress_batch(d, fits)
    assert (status == 0).all()
    for k, (t, S) in enumerate(fits[:10]):
        prep = gcv.Prepared(tprs.design(d, S))
        r, info = gcv.fit(prep, d[:, t])
        err = np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))
        assert err <= RESID_TOL, (t, S, err)


@pytest.mark.parametrize("method", ["dcc.gamma", "hsic.gamma"])
def test_one_shot_batch_equals_staged_graph(lib, method):
    """The one-shot call (bivariate set-up overlapped with the multi-penalty
    fits, launched directly) and the staged form (whole batch prepared, then
    one CUDA-graph replay) run the same kernels on the same designs: their
    records agree bit for bit.  The batch mixes |S| = 0..4, so it has
    pending bivariate designs, additive designs and direct columns."""
    X, triples = workloads.level_batch_500x50(count=600)
    one, st1 = fk.ci_level_batch(X, triples, ci_method=method)
    staged = fk.StagedBatch(X, triples, ci_method=method)
    staged.execute(1)
    two, st2 = staged.collect()
    assert st1["designs"] == st2["designs"] and st1["targets"] == st2["targets"]
    for field in ("p_value", "p_exact", "statistic", "mean", "variance", "status", "flags"):
        assert np.array_equal(one[field], two[field]), field
    # a second one-shot call on the same data reuses the engine's buffers
    again, _ = fk.ci_level_batch(X, triples, ci_method=method)
    assert np.array_equal(again["p_value"], one["p_value"])


# Eleven unequally spaced levels.  On an equally spaced grid the eta matrix is
# symmetric under reversal, half its eigenvectors are antisymmetric, and the
# sign convention (largest-magnitude entry positive) meets exact ties that
# rounding decides, differently in any two implementations.
_LEVELS = np.array([0.0, 1.0, 3.0, 4.5, 7.0, 9.0, 12.0, 15.5, 16.0, 20.0, 23.0])


def _discrete_data(n=300, seed=11):
    """Columns 0 and 1 take 11 values, and their pairs only about 60 distinct
    locations: the bivariate design on {0, 1} has too few unique locations
    for the device Lanczos and is built by the host."""
    rs = np.random.default_rng(seed)
    X = np.empty((n, 8))
    a = rs.integers(0, 11, size=n)
    X[:, 0] = _LEVELS[a]
    X[:, 1] = _LEVELS[(a + rs.integers(0, 6, size=n)) % 11]
    for j in range(2, 8):
        X[:, j] = rs.normal(size=n)
    X[:, 2] += np.sin(X[:, 0])
    X[:, 3] += 0.3 * X[:, 1] + np.tanh(X[:, 2])
    X[:, 6] += np.cos(X[:, 4]) - 0.2 * X[:, 0]
    X[:, 7] += X[:, 5] ** 2 * 0.3
    return np.asfortranarray(X)


def test_host_built_bivariate_design_in_the_one_shot_batch(lib):
    X = _discrete_data()
    pairs = {tuple(int(v) for v in row) for row in X[:, :2]}
    assert 30 <= len(pairs) <= 80  # between the basis size and the device's step count
    triples = [(2, 3, [0, 1]), (4, 6, [0, 1]), (2, 5, [0]), (3, 7, [4, 5]), (2, 6, [0, 1, 4]),
               (6, 7, [0, 4, 5]), (2, 7, []), (3, 6, [1])]
    one, _ = fk.ci_level_batch(X, triples)
    cache = skeleton.ResidualCache(X)
    for k, t in enumerate(triples):
        p = _oracle_p(cache, t)
        assert abs(one["p_value"][k] - p) <= 1e-9, (t, one["p_value"][k], p)
    staged = fk.StagedBatch(X, triples)
    staged.execute(1)
    two, _ = staged.collect()
    assert np.array_equal(one["p_value"], two["p_value"])


@pytest.mark.parametrize("method", ["dcc.perm", "hsic.perm"])
def test_permutation_skeleton_windows_follow_the_sequential_stream(lib, method):
    """p = 12: edges at level 1 and beyond carry several tests, so deletions
    inside a speculative window cut it short and the stream is reset.  The
    skeleton, every p-value and the test counts equal the oracle's strictly
    sequential run."""
    X = workloads.nonlinear_sem(80, 12, 0.25, 21)[0]
    opts = {"ci_method": method, "numCol": 35, "trace_level": "logical",
            "permutation_params": {"replicates": 30, "seed": 7, "include_observed": True}}
    out = fk.fastkpc_compatible_cuda_skeleton(X, 0.1, options=opts)
    ora = skeleton.skeleton(X, 0.1, method, replicates=30, seed=7)
    assert out["n_edgetests"] == ora["n_edgetests"].tolist()
    assert np.array_equal(out["adjacency"], ora["adjacency"])
    got = sorted(zip(out["tasks"]["level"], out["tasks"]["x"], out["tasks"]["y"],
                     map(tuple, out["tasks"]["S"]), out["tasks"]["p_used"]))
    exp = sorted((r["level"], r["x"], r["y"], tuple(r["S"]), r["p_value"]) for r in ora["trace"])
    assert [g[:4] for g in got] == [e[:4] for e in exp]
    assert [g[4] for g in got] == [e[4] for e in exp]


def test_device_smooths_at_n1000_match_oracle(lib):
    """n = 1000: the thin-plate Lanczos runs with leading dimension 1024 (one
    CTA per SM by shared memory), and the geometry kernels, whose n x q
    working matrices no longer fit in shared memory, factor in the arena.
    Univariate, bivariate and additive residuals against the oracle."""
    X = workloads.nonlinear_sem(1000, 12, 0.3, 31)[0]
    fits = [(0, [3, 7]), (5, [1, 2]), (9, [4, 11]), (2, [6]), (8, [0, 5, 10]), (11, [1, 3, 6, 9])]
    resid, lsp, status = fk.regress_batch(X, fits)
    assert (status == 0).all()
    for k, (t, S) in enumerate(fits):
        prep = gcv.Prepared(tprs.design(X, S))
        r, _ = gcv.fit(prep, X[:, t])
        err = np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))
        assert err <= RESID_TOL, (t, S, err)


def test_widest_first_fit_order_changes_no_record(lib):
    """The batched form starts the warp-class fits widest design first
    (|S| = 4, q = 37, before |S| = 3, q = 28); the plain form runs them in
    test order.  With the two widths interleaved, every record agrees bit for
    bit."""
    X, triples = workloads.level_batch_500x50(count=1200)
    wide = [t for t in triples if len(t[2]) == 4]
    narrow = [t for t in triples if len(t[2]) == 3]
    mixed = [t for pair in zip(narrow, wide) for t in pair][:300]
    assert len(mixed) == 300
    batched, st = fk.ci_level_batch(X, mixed)
    plain, _ = fk.ci_level_batch(X, mixed, mode="plain")
    assert np.all(batched["status"] == 0)
    for field in ("p_value", "statistic", "p_exact"):
        assert np.array_equal(batched[field], plain[field]), field


@pytest.mark.parametrize("method", ["dcc.gamma", "hsic.gamma", "dcc.perm"])
def test_empty_batches_return_no_records(lib, method):
    """A level with no tests, a regression with no fits and a statistic call
    with no pairs succeed and return nothing; the staged form, which captures
    a launch sequence, rejects an empty batch."""
    X, _ = workloads.level_batch_500x50(count=1)
    kw = {"seed": 3} if method.endswith("perm") else {}
    for mode in ("batched", "plain"):
        rec, st = fk.ci_level_batch(X, [], ci_method=method, mode=mode, **kw)
        assert all(len(v) == 0 for v in rec.values())
        assert st["pairs"] == 0 and st["kernel_launches"] == 0
    resid, lsp, status = fk.regress_batch(X, [])
    assert resid.shape == (X.shape[0], 0) and status.shape == (0,)
    perms = np.zeros((0, 100, X.shape[0]), dtype=np.int32) if method.endswith("perm") else None
    out = fk.stat_batch(X[:, :4], [], ci_method=method, permutations=perms, **kw)
    assert all(len(v) == 0 for v in out.values())
    with pytest.raises(fk.FkpcError) as e:
        fk.StagedBatch(X, [], ci_method=method, **kw)
    assert e.value.status == 1


def test_near_exact_fit_keeps_a_positive_rss(lib):
    """Variable 7 of the n=351, p=48 SEM with seed 80 is almost exactly a
    smooth of variable 34 (RSS about 4e-13 against |y|^2 = 350).  RSS formed
    as |y|^2 - 2 g'g + |Wg|^2 cancels to rounding noise there; the fit forms
    it as |y - Q Q'y|^2 + |Q'y - W g|^2 and must succeed, with the oracle's
    residual to within 1e-12 of max |y| (the residual itself is at the
    rounding level of y, so a relative bar on it does not apply)."""
    X, _ = workloads.nonlinear_sem(351, 48, 0.1, 80, max_in_degree=8)
    resid, lsp, status = fk.regress_batch(X, [(7, [34])])
    assert status[0] == 0
    prep = gcv.Prepared(tprs.design(X, [34]))
    r, info = gcv.fit(prep, X[:, 7])
    assert info["rss"] > 0.0
    assert np.max(np.abs(resid[:, 0] - r)) <= 1e-12 * np.max(np.abs(X[:, 7]))
    rec, _ = fk.ci_level_batch(X, [(7, 12, [34]), (12, 7, [34])], ci_method="dcc.gamma")
    assert np.all(rec["status"] == 0)


@pytest.mark.parametrize("method", ["dcc.gamma", "hsic.gamma"])
def test_schedule_tunings_change_no_record(lib, method):
    """fkpc_set_tuning changes how a level batch is laid out -- deferral
    threshold, statistics beside the continuation or after every fit,
    Lanczos CTAs per SM -- never a record: one-shot and staged forms give
    bit-identical records under each setting."""
    X, triples = workloads.level_batch_500x50(count=600)
    base = fk.get_tuning(0)
    try:
        ref, _ = fk.ci_level_batch(X, triples, ci_method=method)
        for change in ({"split_statistics": 0}, {"defer_evaluations": 0}, {"defer_evaluations": 40},
                       {"lowrank_ctas_per_sm": 1, "tprs_ctas_per_sm": 1},
                       {"lowrank_ctas_per_sm": 3, "tprs_ctas_per_sm": 3}):
            fk.set_tuning(0, **{**base, **change})
            rec, _ = fk.ci_level_batch(X, triples, ci_method=method)
            batch = fk.StagedBatch(X, triples, ci_method=method)
            batch.execute(1)
            srec, _ = batch.collect()
            for r in (rec, srec):
                for f in ("p_value", "p_exact", "statistic", "mean", "variance", "status", "flags"):
                    assert np.array_equal(np.nan_to_num(r[f]), np.nan_to_num(ref[f])), (change, f)
        with pytest.raises(fk.FkpcError):
            fk.set_tuning(0, lowrank_ctas_per_sm=9)
    finally:
        fk.set_tuning(0, **base)


def test_block_and_single_vector_lanczos_in_one_batch(lib):
    """Bivariate designs with at least 120 unique locations (and a leading
    dimension up to 512) take the block Lanczos; the design on {0, 1} below
    has 95 (two columns of 10 levels each) and takes the single-vector run in
    the same batch.  Residuals of both against the oracle."""
    rs = np.random.default_rng(13)
    n = 300
    X = rs.normal(size=(n, 6))
    lv = np.array([0.0, 1.1, 2.5, 3.2, 4.8, 6.0, 7.7, 9.1, 10.4, 12.9])
    X[:, 0] = lv[rs.integers(0, 10, size=n)]
    X[:, 1] = lv[rs.integers(0, 10, size=n)] * 0.7 + 0.13
    X[:, 2] += np.sin(X[:, 0]) + 0.2 * X[:, 1]
    X[:, 5] += np.tanh(X[:, 3]) - 0.1 * X[:, 0]
    X = np.asfortranarray(X)
    assert len({tuple(r) for r in X[:, :2]}) == 95
    fits = [(2, [0, 1]), (5, [0, 1]), (2, [3, 4]), (5, [3, 4]), (0, [2, 5]), (4, [1, 3])]
    resid, lsp, status = fk.regress_batch(X, fits)
    assert (status == 0).all()
    for k, (t, S) in enumerate(fits):
        prep = gcv.Prepared(tprs.design(X, S))
        r, _ = gcv.fit(prep, X[:, t])
        err = np.max(np.abs(resid[:, k] - r)) / np.max(np.abs(r))
        assert err <= RESID_TOL, (t, S, err)
