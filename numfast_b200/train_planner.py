"""Train the learned planner on engine-generated samples and write planner_weights.npz.

    python -m numfast_b200.train_planner --samples 200000 --timed-every 20 --out numfast_b200/planner_weights.npz

Every sample is one input of the mixed stream (numfast_b200.planner.draw_specs, seed
--seed): its sketch, the exact distinct count the group-by returns, and -- for every
--timed-every-th sample -- the device time of each of the four strategies, whose argmin
is the class label.  The network is trained on the GPU by the library's forward / loss /
backward / Adam kernels.  A held-out slice of the timed samples measures how often the
pick matches the fastest strategy and the time lost against always choosing it, next to
the fixed planner's loss on the same samples.
"""

import argparse
import json
import sys
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=200_000)
    ap.add_argument("--timed-every", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--out", default=None)
    ap.add_argument("--data", default=None, help="reuse / write the collected samples (.npz)")
    ap.add_argument("--report", default=None)
    args = ap.parse_args()
    from numfast_b200 import planner as PL

    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    t0 = time.time()
    if args.data and __import__("os").path.exists(args.data):
        z = np.load(args.data)
        data = {k: z[k] for k in ("features", "distinct", "times")}
        specs_meta = None
    else:
        specs = PL.draw_specs(args.samples, args.seed)
        data = PL.collect(specs, timed_every=args.timed_every, log=log)
        specs_meta = specs
        if args.data:
            np.savez_compressed(args.data, **data)
    t_collect = time.time() - t0
    timed = np.flatnonzero(~np.isnan(data["times"]).any(axis=1))
    rng = np.random.default_rng(args.seed)
    held = rng.choice(timed, size=max(1, len(timed) // 5), replace=False)
    train_mask = np.ones(len(data["distinct"]), bool)
    train_mask[held] = False
    tr = {k: v[train_mask] for k, v in data.items()}
    t1 = time.time()
    params, mu, sd, hist = PL.train(tr, epochs=args.epochs, log=log)
    t_train = time.time() - t1
    out = PL.predict(params, mu, sd, data["features"][held])
    pick = np.argmax(out[:, 1:], axis=1)
    tt = data["times"][held]
    best = np.argmin(tt, axis=1)
    t_best = tt[np.arange(len(held)), best].sum()
    t_pick = tt[np.arange(len(held)), pick]
    # An infeasible dense pick falls back to the fixed planner at run time; count it as
    # the sort time here (the fixed planner's choice for spans the dense family rejects).
    t_pick = np.where(np.isfinite(t_pick), t_pick, tt[:, 3]).sum()
    pred = 2.0 ** (np.clip(out[:, 0], 0, 1) * 32.0) - 1.0
    true = data["distinct"][held].astype(np.float64)
    rel = np.abs(np.log2((pred + 1.0) / (true + 1.0)))
    report = {"samples": int(len(data["distinct"])), "timed": int(len(timed)), "held_out": int(len(held)),
              "collect_s": t_collect, "train_s": t_train, "final_loss": hist[-1],
              "pick_accuracy": float(np.mean(pick == best)),
              "held_time_ratio_pick_over_best": float(t_pick / t_best),
              "distinct_log2_error_median": float(np.median(rel)),
              "distinct_log2_error_p90": float(np.quantile(rel, 0.9)),
              "label_share": [float(np.mean(best == j)) for j in range(4)]}
    log(json.dumps(report))
    if args.out:
        PL.save(args.out, params, mu, sd, min_confidence=0.0, meta=report)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    del specs_meta


if __name__ == "__main__":
    main()
