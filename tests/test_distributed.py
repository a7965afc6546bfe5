"""The sharded skeleton's host logic on CPU ranks (gloo, world size 2).

No GPU: the level evaluator is replaced by a deterministic stand-in whose
p-value depends only on (x, y, S), so the same skeleton must come out of one
process and of two ranks that each evaluate half of every level and gather
the records.  The library plans and replays every level itself
(fkpc_skeleton_run_custom) and uses no device on this path.
"""
import ctypes
import os
import socket

import numpy as np
import pytest

import fastkpc_b200 as fk
from fastkpc_b200 import distributed


def _fake_p(x, y, S):
    a, b = min(x, y), max(x, y)
    h = (a * 7919 + b * 104729 + sum((k + 3) * (v + 1) * 2654435761 for k, v in enumerate(sorted(S)))) % 1000003
    base = (h % 1000) / 1000.0
    return base * (0.35 if (a + b) % 3 else 1.0)  # a third of the pairs depend more weakly on S


def _fake_evaluate(tests):
    out = (fk.CiRecord * max(1, len(tests)))()
    for k, (x, y, S) in enumerate(tests):
        p = _fake_p(x, y, S)
        out[k].p_value = p
        out[k].p_exact = p
    return out


def _data(p=12, n=60):
    return np.asfortranarray(np.random.default_rng(0).normal(size=(n, p)))


OPTS = {"numCol": 35, "trace_level": "logical"}


def _single_process():
    X = _data()
    _, labels, o, method = fk._skeleton_setup(X, 0.1, None, OPTS)

    def level_eval(user, level, x, y, s_offsets, s_values, count, out):
        tests = [(x[i], y[i], [s_values[k] for k in range(s_offsets[i], s_offsets[i + 1])]) for i in range(count)]
        recs = _fake_evaluate(tests)
        for i in range(count):
            out[i] = recs[i]
        return 0
    return fk._run_skeleton(X, 0.1, labels, o, method, fk.LEVEL_EVALUATOR(level_eval))


def _rank_main(rank, world, port, queue):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = distributed.sharded_skeleton(_data(), 0.1, options=OPTS, evaluate=_fake_evaluate)
        queue.put((rank, out["adjacency"].tolist(), out["pMax"].tolist(), out["sepsets"], out["n_edgetests"],
                   out["tasks"]["p_used"].tolist()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_keeps_cohorts_whole_and_covers_every_test():
    tests = [(i % 7, (i + 3) % 11, sorted({i % 5, (i * 3) % 9})) for i in range(200)]
    parts = distributed.partition_tests(tests, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(tests)))
    owner = {}
    for r, idx in enumerate(parts):
        for i in idx:
            key = tuple(tests[i][2])
            assert owner.setdefault(key, r) == r
    assert distributed.partition_tests(tests, 3) == parts  # deterministic


def test_sharded_skeleton_equals_single_process_on_two_gloo_ranks(lib_built):
    import torch.multiprocessing as mp
    ref = _single_process()
    assert sum(ref["n_edgetests"]) > 0 and len(ref["n_edgetests"]) >= 3
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for pr in procs:
        pr.start()
    results = [queue.get(timeout=120) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, adj, pmax, sepsets, n_edgetests, p_used in results:
        assert adj == ref["adjacency"].tolist()
        assert pmax == ref["pMax"].tolist()
        assert sepsets == ref["sepsets"]
        assert n_edgetests == ref["n_edgetests"]
        assert p_used == ref["tasks"]["p_used"].tolist()
