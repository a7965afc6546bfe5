"""The skeleton on several GPUs: each level's CI tests split across ranks.

Tests of one skeleton level are independent given the adjacency at the start
of the level.  ``sharded_skeleton`` runs ``fkpc_skeleton_run_custom`` on every
rank of a ``torch.distributed`` process group (one process per GPU, NCCL or
gloo).  The library plans each level identically on every rank and calls back
here with the level's tests.  Each rank evaluates its share -- whole same-S
cohorts, so no conditioning-set design is built twice -- on its own GPU
through a session (fkpc_session_load once, fkpc_session_evaluate per
level), so the rank's design cache lives across levels.  The 48-byte records are then
all-gathered on the host, and the full level is handed back for the canonical
replay (pMax, sepsets, deletions), which every rank performs identically.  No
collective touches the device data path: the only exchange is the gather of
records, once per level.

The batched gamma methods only: the permutation methods consume one seeded
R stream in pcalg order, test by test, and stay on one GPU.
"""
import ctypes

import numpy as np

import fastkpc_b200 as fk

# Relative cost of one test by |S| (design set-up plus two GCV searches),
# measured on the 500 x 50 level batch; used only to balance the ranks.
_TEST_COST = {0: 0.05, 1: 1.0, 2: 3.0, 3: 6.0, 4: 9.0}


def _test_cost(size):
    return _TEST_COST.get(size, 2.5 * size)


def partition_tests(tests, world):
    """Indices of ``tests`` for each rank.  Tests sharing S stay on one rank
    (the design is built once); cohorts go, largest estimated cost first, to
    the least-loaded rank (ties to the lower rank).  Deterministic, so every
    rank computes the same split."""
    cohorts = {}
    for i, t in enumerate(tests):
        cohorts.setdefault(tuple(int(v) for v in t[2]), []).append(i)
    order = sorted(cohorts.items(), key=lambda kv: (-_test_cost(len(kv[0])) * len(kv[1]), kv[0]))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for S, idx in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].extend(idx)
        load[r] += _test_cost(len(S)) * len(idx)
    for r in out:
        r.sort()
    return out


def level_batch_evaluator(X, options):
    """Evaluate a list of tests on this rank's GPU with ``options`` (an
    ``fkpc_options``): returns a ctypes array of ``CiRecord``.  The data is
    loaded once (a session), so the designs built for one level serve every
    later level; ``evaluate.stats`` collects each call's stage stats."""
    session = fk.Session(X, device=options.device)

    def evaluate(tests):
        if not tests:
            return (fk.CiRecord * 1)()
        out, st = session.evaluate_raw(tests, options)
        evaluate.stats.append(st)
        return out
    evaluate.stats = []
    evaluate.session = session
    return evaluate


def sharded_skeleton(data, alpha, labels=None, options=None, group=None, evaluate=None):
    """``fastkpc_compatible_cuda_skeleton`` with each level's tests split
    across the ranks of ``group`` (the default process group when None).
    Every rank must call it with the same data and options; every rank
    returns the same result.  ``options["device"]`` is this rank's GPU.
    ``evaluate`` (tests -> sequence of ``CiRecord``) replaces the GPU
    evaluation, e.g. for tests of the host logic.  The result's
    ``summary["rank_stats"]`` lists this rank's stage stats per level when
    the GPU evaluator ran."""
    import torch.distributed as dist

    X, labels, o, method = fk._skeleton_setup(data, alpha, labels, options)
    if method not in ("dcc.gamma", "hsic.gamma") or o.mode != fk.MODES["batched"]:
        raise ValueError("the sharded skeleton serves the batched gamma methods (dcc.gamma, hsic.gamma)")
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if evaluate is None:
        evaluate = level_batch_evaluator(X, o)
    failures = []
    rec_size = ctypes.sizeof(fk.CiRecord)

    def level_eval(user, level, x, y, s_offsets, s_values, count, out):
        tests = [(int(x[i]), int(y[i]), [int(s_values[k]) for k in range(s_offsets[i], s_offsets[i + 1])])
                 for i in range(count)]
        mine = partition_tests(tests, world)[rank]
        payload = None
        try:
            recs = evaluate([tests[i] for i in mine])
            payload = b"".join(bytes(recs[k]) for k in range(len(mine)))
        except Exception as exc:  # every rank still joins the gather below
            failures.append(exc)
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine, payload), group=group)
        if any(g[1] is None for g in gathered):
            return 3  # FKPC_STATUS_NUMERIC: some rank could not evaluate its share
        for idx, blob in gathered:
            for k, i in enumerate(idx):
                ctypes.memmove(ctypes.addressof(out[i]), blob[k * rec_size:(k + 1) * rec_size], rec_size)
        return 0

    callback = fk.LEVEL_EVALUATOR(level_eval)
    try:
        out = fk._run_skeleton(X, alpha, labels, o, method, callback)
        out["summary"]["rank_stats"] = list(getattr(evaluate, "stats", []))
        return out
    except fk.FkpcError:
        if failures:
            raise failures[0]
        raise
