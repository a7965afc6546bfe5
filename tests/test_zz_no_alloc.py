"""The allocation-free exact dCov entry point against the allocating one (B200).

``fkpc_dcov_gamma_noalloc`` takes device buffers from the caller (here torch
tensors) and keeps its scratch in a fixed device array inside the library.
Its records must agree with ``fkpc_stat_batch``'s exact-screen values on the
same residuals, on two calls in a row (the second reuses the scratch the
first left behind).  Tolerance 1e-12, the tests' statistic tolerance.
This file is collected last so that it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

import fastkpc_b200 as fk

pytestmark = pytest.mark.gpu

TOL = 1e-12

_RECORD = np.dtype([("p_value", "<f8"), ("p_exact", "<f8"), ("statistic", "<f8"), ("mean", "<f8"),
                    ("variance", "<f8"), ("status", "<i4"), ("flags", "<u4")])


def _pool(n, m, seed):
    rs = np.random.default_rng(seed)
    R = rs.normal(size=(n, m))
    for j in range(1, m, 3):
        R[:, j] = np.tanh(R[:, j - 1]) * rs.uniform(0.1, 1.0) + R[:, j]
    return np.asfortranarray(R)


def _noalloc(R, pairs, torch):
    n, m = R.shape
    dev = torch.device("cuda", 0)
    # column-major n x m: the transpose's row-major storage
    resid = torch.from_numpy(np.ascontiguousarray(R.T)).to(dev)
    flat = torch.tensor(np.asarray(pairs, dtype=np.int32).reshape(-1), device=dev)
    out = torch.zeros(len(pairs) * _RECORD.itemsize, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = fk.load_library().fkpc_dcov_gamma_noalloc(ctypes.c_void_p(resid.data_ptr()), n, m,
                                                   ctypes.c_void_p(flat.data_ptr()), len(pairs),
                                                   ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    fk._check(rc)
    return np.frombuffer(out.cpu().numpy().tobytes(), dtype=_RECORD)


@pytest.mark.parametrize("n,m,seed", [(500, 24, 3), (1200, 9, 5)])
def test_noalloc_matches_stat_batch_twice(lib_built, n, m, seed):
    torch = pytest.importorskip("torch")
    R = _pool(n, m, seed)
    pairs = [(a, b) for a in range(m) for b in range(a + 1, m)]
    ref = fk.stat_batch(R, pairs, ci_method="dcc.gamma")
    for _ in range(2):
        got = _noalloc(R, pairs, torch)
        assert (got["status"] == 0).all()
        assert np.all(np.abs(got["p_value"] - ref["p_exact"]) <= TOL)
        assert np.array_equal(got["p_value"], got["p_exact"])
        exact = (ref["flags"] & fk.FLAG_GUARDED) == 0
        assert exact.any()
        for f in ("statistic", "mean", "variance"):
            assert np.allclose(got[f][exact], ref[f][exact], rtol=TOL, atol=0.0), f
        assert np.all(np.abs(got["p_value"][exact] - ref["p_value"][exact]) <= TOL)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib_built):
    torch = pytest.importorskip("torch")
    with pytest.raises(fk.FkpcError, match="4096"):
        _noalloc(_pool(4097, 2, 1), [(0, 1)], torch)
    with pytest.raises(fk.FkpcError, match="scratch"):
        _noalloc(_pool(4000, 300, 1), [(0, 1)], torch)
    # the entry point still works after the rejected calls
    R = _pool(300, 4, 2)
    got = _noalloc(R, [(0, 1), (2, 3)], torch)
    ref = fk.stat_batch(R, [(0, 1), (2, 3)], ci_method="dcc.gamma")
    assert np.all(np.abs(got["p_value"] - ref["p_exact"]) <= TOL)


def test_noalloc_reports_pairs_outside_the_columns(lib_built):
    torch = pytest.importorskip("torch")
    R = _pool(400, 6, 7)
    # the kernels clamp the bad indices before any read, then the call fails
    for bad in ([(0, 1), (2, 6)], [(-1, 3), (4, 5)]):
        with pytest.raises(fk.FkpcError, match=r"outside \[0, m\)"):
            _noalloc(R, bad, torch)
    pairs = [(0, 1), (2, 3), (4, 5)]
    got = _noalloc(R, pairs, torch)
    ref = fk.stat_batch(R, pairs, ci_method="dcc.gamma")
    assert np.all(np.abs(got["p_value"] - ref["p_exact"]) <= TOL)


def test_noalloc_empty_call_does_no_work(lib_built):
    # count == 0: success with no device work, like the other entry points
    rc = fk.load_library().fkpc_dcov_gamma_noalloc(None, 100, 4, None, 0, None, None)
    assert rc == 0
    rc = fk.load_library().fkpc_dcov_gamma_noalloc(None, 100, 4, None, -1, None, None)
    assert rc == 1
