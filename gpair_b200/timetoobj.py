"""CG time-to-objective: wall time until a reconstruction reaches the plain
method's converged objective.

For one problem:
  plain      CG from the flat prior with the reference's line search, run for
             `iters` iterations; its converged objective J* is the lowest J it
             reached. target = J* (1 + tol), tol = 1e-4 by default.
  T_plain    the same run again, stopped on the device as soon as the current
             image has J <= target (gpair_cg_params.target_J).
  T_batch    flat start, batched line search, same target.
  T_warm     features + network inference + CG with the batched line search
             from the predicted image, same target; if it does not reach the
             target within `iters` iterations the flat-start batched run is
             added (the sequential fallback) and counted.
  T_race     the flat-start fallback runs concurrently from t = 0 in a second
             context (own stream) while the features, the network and the
             warm-started CG run in the first; the first run to reach the
             target sets a shared device flag that ends the other at its next
             iteration (gpair_cg_params.stop_flag). Time until both returned.
All times are host wall clock around the public calls, each call synchronised
(gpair_cg_run returns after the device finished). The CUDA graphs of both line
searches are captured before any timed run.
"""
from __future__ import annotations

import threading
import time
from typing import Dict, List, Optional

import numpy as np

from . import api


def _timed_cg(rec, start, iters, line_search, target, method=2):
    rec.set_image(start)
    t0 = time.perf_counter()
    out = rec.cg(iters, method=method, line_search=line_search, target_J=target)
    return time.perf_counter() - t0, out


def race(rec: api.Reconstructor, rec2: api.Reconstructor, p: api.Problem, net, iters: int, target: float,
         flag: api.StopFlag, rec3: Optional[api.Reconstructor] = None, method: int = 2) -> Dict:
    """Warm start in `rec` against the flat prior in `rec2` (both hold problem p).
    With `rec3` (also holding p), a third runner starts from the flat prior with
    the Fletcher-Reeves beta: on ill-conditioned problems the beta rule moves
    the iterations to the target by large factors either way, so each problem
    takes whichever runner arrives first."""
    import gpair_b200 as g
    from .warmstart import features, warm_start
    flag.reset()
    res: Dict = {}

    def flat(r, key, method):
        r.set_image(p.start_image())
        res[key] = r.cg(iters, method=method, line_search=g.LS_BATCH, target_J=target, stop_flag=flag.ptr)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=flat, args=(rec2, "flat", method))]
    if rec3 is not None:
        threads.append(threading.Thread(target=flat, args=(rec3, "flat_fr", 1)))
    for th in threads:
        th.start()
    img = warm_start(net, rec, p, features(rec, p))
    rec.set_image(img)
    warm = rec.cg(iters, method=method, line_search=g.LS_BATCH, target_J=target, stop_flag=flag.ptr)
    for th in threads:
        th.join()
    dt = time.perf_counter() - t0
    winner = "warm" if warm["reached"] else "none"
    for key in ("flat", "flat_fr"):
        if winner == "none" and key in res and res[key]["reached"]:
            winner = key
    out = {"race_s": dt, "race_winner": winner, "race_warm_iters": warm["iterations"],
           "race_flat_iters": res["flat"]["iterations"]}
    if "flat_fr" in res:
        out["race_flat_fr_iters"] = res["flat_fr"]["iterations"]
    return out


def evaluate(rec: api.Reconstructor, p: api.Problem, net=None, iters: int = 1000, tol: float = 1e-4,
             batch_iters: Optional[int] = None, objective_from: str = "plain",
             rec2: Optional[api.Reconstructor] = None, flag: Optional[api.StopFlag] = None,
             rec3: Optional[api.Reconstructor] = None, method: int = 2) -> Dict:
    """objective_from "plain": J* from the reference line search (the headline
    comparison); "batch": J* from the batched line search run for batch_iters
    iterations from the flat prior (isolates what the network adds). `method`
    is the direction of the batched, warm and race runs (2: PR+ CG, 4:
    projected L-BFGS); plain CG is always PR+ with the reference's search."""
    import gpair_b200 as g
    from .warmstart import features, warm_start
    rec.set_problem(p)
    start = p.start_image()
    bi = batch_iters or iters
    # capture both line-search graphs outside the timed runs (one CUDA graph per mode is cached)
    for ls, m in ((g.LS_WOLFE, 2), (g.LS_BATCH, method)):
        rec.set_image(start)
        rec.cg(1, method=m, line_search=ls)
    rec.set_image(start)
    if objective_from == "plain":
        ref = rec.cg(iters, method=2, trace=True, line_search=g.LS_WOLFE)
    else:
        ref = rec.cg(bi, method=method, trace=True, line_search=g.LS_BATCH)
    Jstar = float(np.min(ref["trace_J"][:ref["iterations"]]))
    target = Jstar * (1.0 + tol) if Jstar > 0 else Jstar * (1.0 - tol)
    res = {"width": p.width, "nuv": p.nuv, "J_star": Jstar, "target": target, "objective_from": objective_from}
    if objective_from == "plain":
        t_plain, o_plain = _timed_cg(rec, start, iters, g.LS_WOLFE, target)
        res.update({"plain_s": t_plain, "plain_iters": o_plain["iterations"], "plain_reached": o_plain["reached"]})
    t_batch, o_batch = _timed_cg(rec, start, bi, g.LS_BATCH, target, method)
    res.update({"batch_s": t_batch, "batch_iters": o_batch["iterations"], "batch_reached": o_batch["reached"]})
    if net is not None:
        t0 = time.perf_counter()
        f = features(rec, p)
        img = warm_start(net, rec, p, f)
        t_net = time.perf_counter() - t0
        t_cg, o_warm = _timed_cg(rec, img, bi, g.LS_BATCH, target, method)
        fell_back = not o_warm["reached"]
        t_fb = 0.0
        if fell_back:
            t_fb, _ = _timed_cg(rec, start, bi, g.LS_BATCH, target, method)
        res.update({"warm_s": t_net + t_cg + t_fb, "warm_net_s": t_net, "warm_iters": o_warm["iterations"],
                    "warm_reached": o_warm["reached"], "fallback": fell_back})
        if rec2 is not None and flag is not None:
            rec2.set_problem(p)
            rec2.set_precision(rec_precision(rec))
            rec2.set_image(start)
            rec2.cg(1, method=method, line_search=g.LS_BATCH)  # graph capture outside the timed race
            if rec3 is not None:
                rec3.set_problem(p)
                rec3.set_precision(rec_precision(rec))
                rec3.set_image(start)
                rec3.cg(1, method=1, line_search=g.LS_BATCH)
            res.update(race(rec, rec2, p, net, bi, target, flag, rec3, method))
    return res


def rec_precision(rec: api.Reconstructor) -> int:
    return int(rec._L.gpair_get_precision(rec.h))


def summarize(rows: List[Dict]) -> Dict:
    def tot(k):
        return float(sum(r[k] for r in rows if k in r))

    out = {"problems": len(rows), "batch_s": tot("batch_s"),
           "batch_reached": int(sum(bool(r["batch_reached"]) for r in rows))}
    has_plain = bool(rows) and "plain_s" in rows[0]
    if has_plain:
        out["plain_s"] = tot("plain_s")
        out["plain_reached"] = int(sum(bool(r["plain_reached"]) for r in rows))
        out["speedup_batch_vs_plain"] = out["plain_s"] / max(out["batch_s"], 1e-12)
    if rows and "warm_s" in rows[0]:
        out["warm_s"] = tot("warm_s")
        out["warm_reached"] = int(sum(bool(r["warm_reached"]) for r in rows))
        out["fallbacks"] = int(sum(bool(r["fallback"]) for r in rows))
        out["speedup_warm_vs_batch"] = out["batch_s"] / max(out["warm_s"], 1e-12)
        if "race_s" in rows[0]:
            out["race_s"] = tot("race_s")
            out["race_winners"] = {w: int(sum(r["race_winner"] == w for r in rows))
                                   for w in ("warm", "flat", "flat_fr", "none")}
            out["speedup_race_vs_batch"] = out["batch_s"] / max(out["race_s"], 1e-12)
            if has_plain:
                out["speedup_race_vs_plain"] = out["plain_s"] / max(out["race_s"], 1e-12)
        if has_plain:
            out["speedup_warm_vs_plain"] = out["plain_s"] / max(out["warm_s"], 1e-12)
            out["median_ratio_warm_vs_plain"] = float(np.median([r["plain_s"] / r["warm_s"] for r in rows]))
    # per problem: width, then iterations to the target (negative: not reached
    # within the limit) of plain CG, the batched search and the warm start
    cols = [k for k in ("plain", "batch", "warm") if f"{k}_iters" in (rows[0] if rows else {})]
    out["per_problem_iters"] = {"columns": ["width"] + cols,
                                "rows": [[int(r["width"])] + [int(r[f"{k}_iters"]) * (1 if r[f"{k}_reached"] else -1)
                                                              for k in cols] for r in rows]}
    return out


def main(argv=None):
    """Evaluate held-out problems (seeds from gpair_b200.train_warmstart.SEED_HELD_OUT):
    the first n64 at 64x64, the next n128 at 128x128; prints one JSON summary per
    objective definition and writes the per-problem rows with --out."""
    import argparse
    import json
    import gpair_b200 as g
    from .train_warmstart import SEED_HELD_OUT
    from .warmstart import DEFAULT_WEIGHTS, WarmStartNet, training_case
    ap = argparse.ArgumentParser()
    ap.add_argument("--n64", type=int, default=16)
    ap.add_argument("--n128", type=int, default=8)
    ap.add_argument("--iters", type=int, default=1000)
    ap.add_argument("--batch-iters", type=int, default=1500)
    ap.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ap.add_argument("--out", default=None)
    ap.add_argument("--rows", default=None, help="append each problem's row to this JSON-lines file as it finishes")
    ap.add_argument("--method", type=int, choices=[2, 4], default=2,
                    help="direction of the batched, warm and race runs (2 PR+, 4 projected L-BFGS)")
    ap.add_argument("--objectives", nargs="+", choices=["plain", "batch"], default=["plain", "batch"],
                    help="J* definitions to evaluate: plain CG's converged objective (the headline) and/or the "
                         "batched search's own (isolates what the network adds)")
    ap.add_argument("--first", type=int, default=0, help="index of the first held-out problem")
    ap.add_argument("--workload", default=None,
                    help="a named workload (gpair_b200.synth) instead of the held-out warm-start problems: plain "
                         "CG against the batched line search, no network")
    args = ap.parse_args(argv)
    if args.workload:
        p = api.workload_problem(args.workload)
        with g.Reconstructor(0) as rec:
            rec.set_precision(g.PREC_SPLIT16)
            row = evaluate(rec, p, None, iters=args.iters, batch_iters=args.batch_iters, objective_from="plain",
                           method=args.method)
        print("SUMMARY", json.dumps(row), flush=True)
        return
    net = WarmStartNet.load(args.weights)
    rows = {k: [] for k in args.objectives}
    flag = api.StopFlag()
    with g.Reconstructor(0) as rec, g.Reconstructor(0) as rec2:
        rec.set_precision(g.PREC_SPLIT16)
        for k in range(args.first, args.first + args.n64 + args.n128):
            width = 64 if k - args.first < args.n64 else 128
            p = training_case(SEED_HELD_OUT + k, width).problem
            for obj in args.objectives:
                r = evaluate(rec, p, net, iters=args.iters, batch_iters=args.batch_iters if obj == "batch" else None,
                             objective_from=obj, rec2=rec2, flag=flag, method=args.method)
                r["seed"] = SEED_HELD_OUT + k
                rows[obj].append(r)
                if args.rows:
                    with open(args.rows, "a") as f:
                        f.write(json.dumps({"objective": obj, **r}) + "\n")
    flag.close()
    for k in args.objectives:
        print(f"SUMMARY {k}", json.dumps(summarize(rows[k])), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f)


if __name__ == "__main__":
    main()
