"""Achieved bandwidth and FLOP rate of every stage of one criterion + gradient
evaluation, for the named workloads.

    python -m gpair_b200.stage_report [--workloads precision large] [--reps 10]
    python -m gpair_b200.stage_report --workloads large --cg 1 [--method 2] [--line-search 0]
    python -m gpair_b200.stage_report --batch 64 [--iters 30] [--precision 4]

A workload is a named one (gpair_b200.synth.workload) or instance:SEED, one
problem of the many-instance workload (gpair_b200.instances.instance).

With --batch N: N instances of the many-instance workload, autotuned as the
benchmark tunes them, their adjoint split-K lengths set for sharing the GPU
(gpair_set_shared_splits), run as one staged lockstep batch with the batched
line search; prints the device time and the per-launch time of every stage
summed over the run (device timer stamps, gpair_batch_stage_stamps), with the
SM clock sampled during the run.

With --cg N the module instead runs N CG iterations from the flat prior,
driven from the host (every kernel a plain launch, so that a profiler's
launch list shows each one), and prints the evaluation counts: the command
for launch lists of one CG iteration.

Stages and time: `Reconstructor.time_stages` (CUDA events around the stages
queued back to back), split-f16 tensor path.

Bytes per stage are the stage's compulsory traffic, as its kernels move it:

  prep           image + prior read for flux / entropy / max (8 B/px), image
                 read again and the f16 hi/lo operand written (8 B/px)
  vis_data       V2: partial visibilities (8 B per partial entry: one per 128
                 image rows, rounded up to 256), data + inverse
                 error (8 B), visibilities written (16 + 8 B), mock (4 B), uv
                 weight (8 B); T3: indices (16 B), three gathered visibilities
                 (3 x 8 B per partial entry), phasor (8 B), data + error (16 B),
                 mock (8 B), vertex weights written (24 B)
  adj_weights    uv weights + CSR gather of vertex weights (16 B per point +
                 12 B per triangle vertex), then the adjoint's f16 hi/lo weight
                 operand W written (8 B per pixel row per uv point: 8 N nuv)
  grad_finalize  S split partial images read (4 S B/px), image, prior,
                 previous gradient and direction read (16 B/px), data, entropy
                 and full gradient written (12 B/px)
  forward_dft / adjoint_dft  algorithmic FLOPs 4 N^2 nuv + 8 N nuv (TFLOP/s);
                 executed = the MMA work in f16-rate units per algorithmic
                 product: 3 for split-f16 (three f16 products); for
                 split-f16/E4M3 the forward is 2 (one f16 product and two E4M3
                 products at twice the rate), the adjoint 3
"""
from __future__ import annotations

import argparse
import json
import os

from . import api


def stage_bytes(p: api.Problem, splits: int, row_tiles: int) -> dict:
    N, K, T = p.width, p.nuv, p.nbis
    px = N * N
    return {
        "prep": 16 * px,
        "vis_data": p.npow * (8 * row_tiles + 8 + 24 + 4 + 8) + T * (16 + 24 * row_tiles + 8 + 16 + 8 + 24),
        "adj_weights": 16 * K + 12 * 3 * T + 8 * N * K,
        "grad_finalize": (4 * splits + 28) * px,
    }


def problem(name: str) -> api.Problem:
    """A named workload, or instance:SEED of the many-instance workload."""
    if name.startswith("instance:"):
        from .instances import instance
        return instance(int(name.split(":", 1)[1]))
    return api.workload_problem(name)


def batch_report(n: int, iters: int, precision: int, tune: str = "all", prep_passes=(0,)) -> list:
    """Stage breakdown of a staged lockstep batch of n many-instance problems,
    one report per trial-prep pass count (0: the batch's own choice).
    tune "all": every instance's precision path, tile and split-K autotuned
    alone; "splits": `precision` and single CTAs for all (one class per
    contraction), only the split-K length tuned."""
    from .clocks import ClockSampler
    from .instances import instances
    ps = instances(n)
    recs = [api.Reconstructor(0) for _ in ps]
    out = []
    try:
        for r, p in zip(recs, ps):
            if tune == "splits":
                r.set_tc_pair(False)
            r.set_problem(p)
            r.set_precision(precision)
            r.set_image(p.start_image())
        flags = api.TUNE_SPLITS | api.TUNE_CACHE | api.TUNE_BATCHED
        if tune == "all":
            flags |= api.TUNE_PRECISION | api.TUNE_TILE
        for r in recs:
            r.autotune(flags, reps=2)
        api.shared_splits(recs)
        for passes in prep_passes:
            with api.Batch(recs, line_search=api.LS_BATCH, stamps=True, prep_passes=passes) as b:
                for r, p in zip(recs, ps):
                    r.set_image(p.start_image())
                b.run(1)  # first launch
                b.stage_times_us(reset=True)
                for r, p in zip(recs, ps):
                    r.set_image(p.start_image())
                sampler = ClockSampler(0)
                sampler.start()
                res = b.run(iters)
                clocks = sampler.stop()
                dev_ms = recs[0].last_run_stats()[0]
                flops = sum(r.last_run_stats()[1] for r in recs)
                stages = b.stage_times_us()
                total = sum(v for k, v in stages.items() if k != "batched_evaluations")
                out.append({
                    "instances": n, "iterations": iters, "precision": precision, "tune": tune,
                    "layout": b.grouped, "prep_passes": b.prep_passes, "device_ms": dev_ms,
                    "tflops": flops / (dev_ms * 1e-3) / 1e12, "clocks": clocks,
                    "all_ok": all(o["status"] == 0 for o in res), "J": [o["J"] for o in res],
                    "stage_us": stages,
                    "stage_share": {k: v / total for k, v in stages.items() if k != "batched_evaluations"},
                    "timing": "device timer stamps after every launch (one small timer kernel each), summed over "
                              "the run"})
    finally:
        for r in recs:
            r.close()
    return out


def report(name: str, reps: int = 10, pair: bool = False, precision: int = api.PREC_SPLIT16) -> dict:
    from .clocks import ClockSampler
    p = problem(name)
    with api.Reconstructor(0) as rec:
        rec.set_problem(p)
        rec.set_precision(precision)
        rec.set_tc_pair(pair)
        rec.set_image(p.start_image())
        rec.criterion()
        rec.gradient()
        sampler = ClockSampler(0)
        sampler.start()
        st = rec.time_stages(reps=reps)
        for _ in range(4):  # long enough for a few 200 ms clock samples
            st2 = rec.time_stages(reps=reps)
            st = {k: min(st[k], st2[k]) for k in st}
        clocks = sampler.stop()
    peaks_path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    hbm, tf = 6650.0, 1590.0
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            d = json.load(f)
        hbm, tf = d["hbm_gbs"], d["bf16_tflops"]
    row_tiles = 2 * ((p.width + 255) // 256)  # partial entries of the tensor forward
    splits = _default_splits(p, pair)
    by = stage_bytes(p, splits, row_tiles)
    out = {"workload": name, "precision": precision, "N": p.width, "nuv": p.nuv, "npow": p.npow, "nbis": p.nbis,
           "splits": splits,
           "hbm_peak_gbs": hbm, "tensor_peak_tflops": tf, "clocks": clocks, "cta_pairs": bool(pair),
           "timing": f"CUDA events, stages back to back, best of 5 x {reps} repetitions", "stages": {}}
    for k, ms in st.items():
        row = {"ms": ms}
        if k in by:
            gbs = by[k] / (ms * 1e-3) / 1e9
            row.update({"bytes": by[k], "gbs": gbs, "hbm_frac": gbs / hbm})
        else:
            tfl = p.dft_flops() / (ms * 1e-3) / 1e12
            mult = 2.0 if (precision == api.PREC_SPLIT16F8 and k == "forward_dft") else 3.0
            row.update({"tflops": tfl, "frac": tfl / tf, "executed_frac": mult * tfl / tf})
        out["stages"][k] = row
    return out


def _default_splits(p: api.Problem, pair: bool = False) -> int:
    """Split count of the tensor adjoint as the library chooses it (mirrors gp_tc_splits, f16 operands)."""
    N, K = p.width, p.nuv
    tm, slots = (256, 74) if pair else (128, 148)
    m_pad = -(-N // 256) * 256
    xrows = -(-N // tm) * tm
    k2 = -(-2 * K // 64) * 64
    tiles = (xrows // tm) * (m_pad // 256)
    kb_total = k2 // 64
    want = max(1, min(kb_total, -(-slots // tiles)))
    kb_per = min(64, -(-kb_total // want))
    return -(-kb_total // kb_per)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", nargs="+", default=["precision", "large"])
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--cg", type=int, default=0, help="run this many host-driven CG iterations instead")
    ap.add_argument("--method", type=int, default=2)
    ap.add_argument("--line-search", type=int, default=0, help="0 the reference's search, 1 batched")
    ap.add_argument("--precision", type=int, default=api.PREC_SPLIT16)
    ap.add_argument("--tc-pair", type=int, default=1, help="contractions on CTA pairs (cta_group::2, 1) or single CTAs (0)")
    ap.add_argument("--batch", type=int, default=0, help="stage breakdown of a staged batch of this many instances")
    ap.add_argument("--iters", type=int, default=30, help="CG iterations of the --batch run")
    ap.add_argument("--tune", choices=["all", "splits"], default="all",
                    help="--batch: autotune precision, tile and split-K per instance, or split-K only")
    ap.add_argument("--prep-passes", type=int, nargs="+", default=[0],
                    help="--batch: passes of image rows per trial-prep block, one run each (0: the batch's choice)")
    args = ap.parse_args(argv)
    if args.batch > 0:
        for rep in batch_report(args.batch, args.iters, args.precision, args.tune, args.prep_passes):
            print(json.dumps(rep), flush=True)
        return
    for w in args.workloads:
        if args.cg > 0:
            p = problem(w)
            with api.Reconstructor(0) as rec:
                rec.set_problem(p)
                rec.set_precision(args.precision)
                rec.set_tc_pair(bool(args.tc_pair))
                rec.set_image(p.start_image())
                out = rec.cg(args.cg, method=args.method, line_search=args.line_search, host_loop=1)
            print(json.dumps({"workload": w, "iterations": out["iterations"], "criterion_evals": out["criterion_evals"],
                              "grad_evals": out["grad_evals"], "J": out["J"]}), flush=True)
            continue
        print(json.dumps(report(w, args.reps, bool(args.tc_pair), args.precision)), flush=True)


if __name__ == "__main__":
    main()
