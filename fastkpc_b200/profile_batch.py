"""Run one prepared level batch for profiling (ncu / nsight).

    python -m fastkpc_b200.profile_batch [--count 4096] [--method dcc.gamma] [--repeats 1]

Prepares the single-level CI batch (n=500, p=50 nonlinear SEM, |S| uniform on
0..4), replays its captured launch sequence ``repeats`` times after one
warm-up replay, collects and checks the records, and prints the per-stage
device times.  Exit status 0 only when every record is valid.
"""
import argparse
import json
import sys

import numpy as np

import fastkpc_b200 as fk
from fastkpc_b200 import workloads


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--method", default="dcc.gamma", choices=["dcc.gamma", "hsic.gamma"])
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    X, triples = workloads.level_batch_500x50(count=args.count)
    batch = fk.StagedBatch(X, triples, ci_method=args.method, device=args.device)
    batch.execute(1)
    ms = batch.execute(args.repeats)
    recs, st = batch.collect()
    ok = bool(np.all(recs["status"] == 0))
    stages = {}
    for name in ("fit_single", "fit_multi_small", "fit_multi_large", "dcov_components", "dcov_pairs",
                 "lowrank_eigen", "lowrank_pairs"):
        if args.method == "hsic.gamma" and name.startswith(("dcov", "lowrank")):
            continue
        stages[name] = batch.time_stage(name, repeats=2)[0]
    print(json.dumps({"count": args.count, "method": args.method, "repeats": args.repeats, "device_ms": ms,
                      "stages_ms": stages, "fits": st["targets"], "fit_evaluations": st["fit_evaluations"],
                      "fit_iterations": st["fit_iterations"], "lowrank_components": st["lowrank_components"],
                      "lowrank_steps_mean": st["lowrank_steps_mean"], "lowrank_steps_max": st["lowrank_steps_max"],
                      "launches_per_replay": st["kernel_launches"], "ok": ok}))
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
