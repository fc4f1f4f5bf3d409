#!/usr/bin/env python
"""Benchmark of the GPAIR reconstruction hot path on B200.

Workload (default, `--workload large`): the 1024x1024 polychromatic
reconstruction -- 0.02 mas/pixel, a limb-darkened 15 mas disk with 50 Gaussian
spots (+-30 % contrast), 20 telescopes in a 400 m disk (190 baselines), 64 hour
angles x 16 channels: 194,560 V2 points and 1,167,360 closure triangles
(nuv = 195,021 after the reference's uv matcher), seeded synthetic data (the
reference publishes no data set of this size). It is the largest
configuration that fits one GPU (2.5 GB of HBM). The 256x256 "precision"
workload (21,120 V2, 70,400 T3) is reported beside it under `precision_256`.

A step is one plain PR+ nonlinear-CG iteration with the reference's strong
Wolfe line search (criterion + gradient of the current image, direction
update, bracketing/zoom trials, image update), continuing from the previous
step. Metric: algorithmic DFT + adjoint TFLOP/s over the timed steps, i.e.
(criterion + gradient evaluations) x (4 N^2 nuv + 8 N nuv) / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is timed with CUDA events on the library's stream (inputs resident in
HBM, L2 flushed by a 512 MiB write before every step, outside the timed
region); `e2e` times the same steps through the public C ABI with host
buffers: image upload, one CG iteration, image read-back. With N > 1 each rank
runs its own independent reconstruction (replicas, weak scaling); the time is
the max over ranks.

`--impl reference` times the reference's own CPU code path on the host cores:
its cpu.c criterion + gradient (compiled unchanged from the reference's
sources into oracle/_ref) on a bounded sample of the same workload, whose uv
and triangle indices come from the reference's own getoifits.c. That process
never imports the gpair_b200 package and maps none of its libraries.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CG time-to-objective (learned warm-start vs plain) + DFT/grad TFLOP/s, 1 B200"
UNIT = "TFLOP/s (algorithmic DFT+adjoint, plain PR+ CG iterations)"


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


# ----------------------------------------------------------- measurements

LS = {"wolfe": 0, "batch": 1}
# independent contexts' streams should map to distinct hardware queues (default 8)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def _traffic(kernel_key):
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel_key)
    return None


# ------------------------------------------------ the reference's CPU path

def data_modules():
    """The seeded data generator (gpair_b200/synth.py) and its OIFITS tables
    (gpair_b200/oifits.py), loaded as plain modules under a private package
    name: the gpair_b200 package, its ctypes layer and libgpair_b200.so are
    not touched (the reference arm must run none of this project's code on
    its measured path)."""
    name = "_gpair_data_only"
    if name in sys.modules:
        pkg = sys.modules[name]
        return pkg.synth, pkg.oifits
    pkg = types.ModuleType(name)
    pkg.__path__ = [os.path.join(ROOT, "gpair_b200")]
    sys.modules[name] = pkg
    for mod in ("oifits", "synth"):
        spec = importlib.util.spec_from_file_location(f"{name}.{mod}", os.path.join(ROOT, "gpair_b200", f"{mod}.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"{name}.{mod}"] = m
        spec.loader.exec_module(m)
        setattr(pkg, mod, m)
    return pkg.synth, pkg.oifits


def subset_channels(oi, chans, oifits_mod, rows_v2=None, rows_t3=None):
    """The same OIFITS tables restricted to the spectral channels `chans` (and,
    when given, to the record rows `rows_v2` / `rows_t3`)."""
    import numpy as np
    ch = np.asarray(chans)
    M = oifits_mod

    def r(a, rows):
        return a if rows is None else a[rows]

    wv = [M.WavelengthTable(x.insname, x.eff_wave[ch], x.eff_band[ch]) for x in oi.wavelengths]
    v2 = [M.Vis2Table(t.insname, r(t.target_id, rows_v2), r(t.ucoord, rows_v2), r(t.vcoord, rows_v2),
                      r(t.vis2data, rows_v2)[:, ch], r(t.vis2err, rows_v2)[:, ch], r(t.flag, rows_v2)[:, ch])
          for t in oi.vis2]
    t3 = [M.T3Table(t.insname, r(t.target_id, rows_t3), r(t.u1coord, rows_t3), r(t.v1coord, rows_t3),
                    r(t.u2coord, rows_t3), r(t.v2coord, rows_t3), r(t.t3amp, rows_t3)[:, ch],
                    r(t.t3amperr, rows_t3)[:, ch], r(t.t3phi, rows_t3)[:, ch], r(t.t3phierr, rows_t3)[:, ch],
                    r(t.flag, rows_t3)[:, ch]) for t in oi.t3]
    return M.OIFits(wv, v2, t3, oi.target_id)


# CPU sample of a workload: one spectral channel of its data (the middle one)
# and every SAMPLE_HA_STRIDE-th hour angle, indexed by the reference's
# getoifits.c, on a SAMPLE_WIDTH^2 image. The reference's criterion + gradient
# cost is linear in the pixel count and in the V2 and triangle counts, and the
# subset keeps the workload's ratio of triangles to uv points, so the per-FLOP
# rate carries over to the full size. The subset is small enough that one
# process's DFT tables stay in its core's caches (about 1.5 MB at 1024^2), so
# that every host core can run one at once without the steps turning into
# DRAM-bound table gathers.
SAMPLE_WIDTH = 32
SAMPLE_HA_STRIDE = 4


def reference_sample(workload: str, oi=None, width: int = SAMPLE_WIDTH) -> dict:
    """Arrays of the CPU sample, built only by the reference's compiled code:
    getoifits.c for the uv / triangle indices, gpair.c's init_data for the data
    packing, cpu.c's set_model for the prior."""
    import numpy as np
    from oracle import oracle as O
    synth, oifits_mod = data_modules()
    w = synth.workload(workload)
    if oi is None:
        _, oi = synth.make_workload_data(workload)
    nch = len(w.array.wavelengths_m)
    ch = nch // 2
    # records are hour-angle major (synth.make_oifits): keep every SAMPLE_HA_STRIDE-th hour angle
    cfg = w.array
    nbl = cfg.n_tel * (cfg.n_tel - 1) // 2
    ntr = oi.t3[0].t3amp.shape[0] // cfg.n_ha
    ha = np.arange(0, cfg.n_ha, SAMPLE_HA_STRIDE)
    rows_v2 = (ha[:, None] * nbl + np.arange(nbl)[None, :]).ravel()
    rows_t3 = (ha[:, None] * ntr + np.arange(ntr)[None, :]).ravel()
    sub = subset_channels(oi, [ch], oifits_mod, rows_v2, rows_t3)
    ix = O.ref_index(sub)
    data, err, ph, _ = O.ref_init_data(ix["npow"], ix["nbis"], ix["pow"], ix["powerr"], ix["bisamp"],
                                       ix["bisamperr"], ix["bisphs"], ix["bisphserr"], ix["uvpnt"], 1)
    model = O.ref_set_model(width, w.pixellation_mas, 0, 0.0, 1.0)
    data_scale = nch * cfg.n_ha / len(ha)  # full data / sample data
    return {"width": width, "pixellation": w.pixellation_mas, "uv": ix["uv"], "npow": ix["npow"],
            "nbis": ix["nbis"], "data": data, "data_err": err, "phasor": ph, "uvpnt": ix["uvpnt"],
            "sign": ix["sign"], "model": model, "alpha": w.alpha, "full_width": w.image_width, "channels": nch,
            "channel": ch, "data_scale": data_scale,
            "describe": (f"channel {ch + 1} of {nch}, hour angles 1 of {SAMPLE_HA_STRIDE} ({ix['npow']} V2, "
                         f"{ix['nbis']} T3, nuv {ix['nuv']}, indexed by the reference's getoifits.c) on a "
                         f"{width}x{width} image")}


def reference_problem(workload: str, oi=None) -> dict:
    """The whole workload's arrays, built only by the reference's compiled code
    (getoifits.c indices, gpair.c init_data packing, cpu.c set_model prior), at
    the workload's own image size."""
    from oracle import oracle as O
    synth, _ = data_modules()
    w = synth.workload(workload)
    if oi is None:
        _, oi = synth.make_workload_data(workload)
    ix = O.ref_index(oi)
    data, err, ph, _ = O.ref_init_data(ix["npow"], ix["nbis"], ix["pow"], ix["powerr"], ix["bisamp"],
                                       ix["bisamperr"], ix["bisphs"], ix["bisphserr"], ix["uvpnt"], 1)
    model = O.ref_set_model(w.image_width, w.pixellation_mas, 0, 0.0, 1.0)
    return {"width": w.image_width, "pixellation": w.pixellation_mas, "uv": ix["uv"], "npow": ix["npow"],
            "nbis": ix["nbis"], "data": data, "data_err": err, "phasor": ph, "uvpnt": ix["uvpnt"],
            "sign": ix["sign"], "model": model, "alpha": w.alpha}


class _SampleProblem:
    def __init__(self, s):
        self.__dict__.update(s)

    @property
    def nuv(self):
        return int(self.uv.shape[0])

    @property
    def npix(self):
        return self.width * self.width

    def dft_flops(self):
        return 4.0 * self.npix * self.nuv + 8.0 * self.width * self.nuv


_WORKER = {}


def _ref_worker_init(sample):
    """Pool initializer: the reference's cpu.c evaluator on the sample arrays."""
    from oracle import oracle as O
    p = _SampleProblem(sample)
    _WORKER["p"] = p
    _WORKER["ev"] = O.RefEvaluator(p)
    # cpu.c's image2vis prints on every call (gpair1/trunk/cpu.c:460)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)


def _ref_eval(reps):
    """`reps` criterion + gradient evaluations with the reference's cpu.c."""
    import numpy as np
    p, ev = _WORKER["p"], _WORKER["ev"]
    img = np.maximum(p.model, np.float32(1e-8)).astype(np.float32)
    t0 = time.perf_counter()
    for _ in range(reps):
        ev.chi2(img)
        ev.data_gradient(img)
        ev.entropy_gradient(img)
    dt = time.perf_counter() - t0
    return reps * 2 * p.dft_flops(), dt


def cpu_baseline(sample, reps=20):
    """The reference's cpu.c on the sample, one core, in this process."""
    import numpy as np
    from oracle import oracle as O
    p = _SampleProblem(sample)
    ev = O.RefEvaluator(p)
    img = np.maximum(p.model, np.float32(1e-8)).astype(np.float32)
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # cpu.c's image2vis prints on every call
    try:
        t0 = time.perf_counter()
        for _ in range(reps):
            ev.chi2(img)
            ev.data_gradient(img)
            ev.entropy_gradient(img)
        dt = time.perf_counter() - t0
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    flops = reps * 2 * p.dft_flops()
    per_eval = dt / reps
    scale = (sample["full_width"] / p.width) ** 2 * sample["data_scale"]
    return {"value": flops / dt / 1e12, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"reference cpu.c criterion+gradient, {sample['describe']}, {reps} evaluations ({dt:.1f} s)",
            "extrapolated": True,
            "extrapolated_full_evaluation_s": per_eval * scale,
            "extrapolation": (f"per-evaluation time x (full width / sample width)^2 x (full data / sample data) = "
                              f"x{scale:.0f}; the reference's cost is linear in pixels, V2 points and triangles")}


def run_reference(args, rank):
    """The reference arm: the reference's own compiled cpu.c on all host cores,
    on the CPU sample of the workload (see reference_sample)."""
    import multiprocessing as mp
    if rank != 0:
        return
    t_setup = time.perf_counter()
    sample = reference_sample(args.workload)
    t_setup = time.perf_counter() - t_setup
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_worker_init, initargs=(sample,)) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_eval, [1] * cores)
        t0 = time.perf_counter()
        tot = 0.0
        for _ in range(args.steps):
            res = pool.map(_ref_eval, [1] * cores)
            tot += sum(r[0] for r in res)
        dt = time.perf_counter() - t0
    value = tot / dt / 1e12
    synth, _ = data_modules()
    w = synth.workload(args.workload)
    cfg = w.array
    nbl = cfg.n_tel * (cfg.n_tel - 1) // 2
    ntri = cfg.n_tel * (cfg.n_tel - 1) * (cfg.n_tel - 2) // 6 if cfg.triangles == "all" else (
        (cfg.n_tel - 1) * (cfg.n_tel - 2) // 2)
    nch = len(cfg.wavelengths_m)
    maps = _mapped_libraries()
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(args.steps, 1), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (reference cpu.c, float complex)",
           "data": "synthetic (seeded)", "impl": "reference",
           "config": {"workload": (f"{args.workload}: {w.image_width}x{w.image_width} image, "
                                   f"{nbl * cfg.n_ha * nch} V2, {ntri * cfg.n_ha * nch} T3"),
                      "sample": (f"{sample['describe']}; one criterion+gradient evaluation per core per step; "
                                 "throughput extrapolates to the full workload (cost linear in pixels, V2 points "
                                 "and triangles)"),
                      "setup_s": t_setup},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                            "sample": f"{cores} processes x criterion+gradient, {sample['describe']}"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "native_libraries": maps}
    if any("libgpair_b200" in m for m in maps):
        raise RuntimeError("the reference arm mapped this project's library")
    print(json.dumps(out), flush=True)


def _mapped_libraries():
    """Shared objects of this repository mapped into this process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                parts = ln.split()
                if len(parts) >= 6 and parts[-1].endswith(".so") and parts[-1].startswith(ROOT):
                    out.add(os.path.relpath(parts[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


# ----------------------------------------------------------- our arm

def replica_seeds(rank):
    """Seeds of rank `rank`'s replica: the same array and scene on every rank, an own noise seed."""
    return {"scene_seed": 1, "noise_seed": 2 + rank, "array_seed": 3}


def combine_over_ranks(times, work, device=None):
    """Whole-job figures of independent replicas: the slowest rank's times (max) and
    the work of all ranks (sum). The only collective of a run, outside the timed region."""
    import torch
    t = torch.tensor(times, dtype=torch.float64, device=device)
    w = torch.tensor(work, dtype=torch.float64, device=device)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.SUM)
    return [float(x) for x in t.tolist()], [float(x) for x in w.tolist()]


def many_instances(n: int, iters: int, precision: int) -> dict:
    """n independent reconstructions of uneven size (widths 64-256, 500-8,000 uv)
    for `iters` batched-line-search CG iterations each: one after another, all
    at once through gpair_cg_run_many (each context's graph on its own stream),
    (with one precision path and tile layout for all, chosen by timing staged batches,
    and gpair_set_shared_splits: the adjoint split-K lengths for instances that
    share the GPU) and as one graph launch (gpair_batch_run) in three layouts: the staged lockstep
    batch (every stage of an iteration one launch over all instances, every
    contraction one grouped tcgen05 launch per class), the lockstep batch with
    grouped trial forwards only, and every CG loop an independent branch of the
    graph. Host wall clock; problem loading and graph capture are outside the
    timings."""
    import gpair_b200 as g
    from gpair_b200.instances import instances
    ps = instances(n)
    recs = [g.Reconstructor(0) for _ in ps]
    try:
        # sequential baseline: the given precision path on single CTAs, the adjoint split-K
        # length autotuned per instance shape (cached across equal shapes)
        for r, p in zip(recs, ps):
            r.set_tc_pair(False)
            r.set_problem(p)
            r.set_precision(precision)
            r.set_image(p.start_image())
        t0 = time.perf_counter()
        flags = g.api.TUNE_SPLITS | g.api.TUNE_CACHE | g.api.TUNE_BATCHED
        tuned = [r.autotune(flags, reps=2) for r in recs]
        t_tune = time.perf_counter() - t0
        for r, p in zip(recs, ps):
            r.set_image(p.start_image())
        g.cg_many(recs, 1, line_search=g.LS_BATCH)  # builds every graph
        for r, p in zip(recs, ps):
            r.set_image(p.start_image())
        t0 = time.perf_counter()
        for r in recs:
            r.cg(iters, method=2, line_search=g.LS_BATCH)
        t_seq = time.perf_counter() - t0
        flops = sum(r.last_run_stats()[1] for r in recs)
        # run together: one precision path and tile layout for all instances (one class per
        # contraction in a staged batch: 80.2 ms against 82.4 ms with precision and tile
        # autotuned per instance, python -m gpair_b200.stage_report --batch 64 --tune
        # splits|all), chosen by timing a staged batch under each candidate, and the adjoint's
        # K dimension split for the GPU the instances share (gpair_set_shared_splits)
        t0 = time.perf_counter()
        layout = g.api.tune_batch_layout(recs, ps)
        t_layout = time.perf_counter() - t0
        for r, p in zip(recs, ps):
            r.set_image(p.start_image())
        g.cg_many(recs, 1, line_search=g.LS_BATCH)  # rebuilds the graphs
        for r, p in zip(recs, ps):
            r.set_image(p.start_image())
        t0 = time.perf_counter()
        res = g.cg_many(recs, iters, line_search=g.LS_BATCH)
        t_con = time.perf_counter() - t0
        flops_con = sum(r.last_run_stats()[1] for r in recs)
        # one graph launch: staged lockstep, lockstep with grouped forwards only, independent branches
        one = {}
        for mode in ("staged", "forwards_only", "independent"):
            with g.api.Batch(recs, line_search=g.LS_BATCH, independent=(mode == "independent"),
                             forwards_only=(mode == "forwards_only")) as b:
                for r, p in zip(recs, ps):
                    r.set_image(p.start_image())
                b.run(1)  # first launch
                for r, p in zip(recs, ps):
                    r.set_image(p.start_image())
                t0 = time.perf_counter()
                res_b = b.run(iters)
                dt = time.perf_counter() - t0
                one[mode] = {"s": dt, "grouped": b.grouped, "prep_passes": b.prep_passes,
                             "all_ok": all(r_["status"] == 0 for r_ in res_b),
                             "tflops": sum(r.last_run_stats()[1] for r in recs) / max(dt, 1e-12) / 1e12}
        t_one = one["staged"]["s"]
    finally:
        for r in recs:
            r.close()
    return {"instances": n, "iterations": iters,
            "widths": {w: sum(p.width == w for p in ps) for w in (64, 128, 192, 256)},
            "uv_range": [min(p.nuv for p in ps), max(p.nuv for p in ps)],
            "sequential_s": t_seq, "concurrent_s": t_con, "speedup": t_seq / max(t_con, 1e-12),
            "instances_per_s": n / max(t_con, 1e-12), "tflops_concurrent": flops_con / max(t_con, 1e-12) / 1e12,
            "tflops_sequential": flops / max(t_seq, 1e-12) / 1e12,
            "one_launch_s": t_one, "one_launch_speedup": t_seq / max(t_one, 1e-12),
            "tflops_one_launch": one["staged"]["tflops"], "one_launch_grouped": one["staged"]["grouped"],
            "one_launch_prep_passes": one["staged"]["prep_passes"],
            "one_launch_forwards_only_s": one["forwards_only"]["s"],
            "tflops_one_launch_forwards_only": one["forwards_only"]["tflops"],
            "one_launch_independent_s": one["independent"]["s"],
            "tflops_one_launch_independent": one["independent"]["tflops"],
            "all_ok": all(r_["status"] == 0 for r_ in res) and all(v["all_ok"] for v in one.values()),
            "autotune": {"what": ("sequential runs: the bench precision on single CTAs, adjoint split-K per shape; "
                                  "run together: one precision path and tile layout for all, from timed staged-batch "
                                  "runs of each candidate (gpair_b200.api.tune_batch_layout), shared split-K"),
                         "layout": layout, "layout_s": t_layout, "s": t_tune,
                         "tuned": sum(not t["from_cache"] for t in tuned),
                         "fp32_path": sum(t["precision"] == g.PREC_FP32 for t in tuned),
                         "split16_path": sum(t["precision"] == g.PREC_SPLIT16 for t in tuned),
                         "split16f8_path": sum(t["precision"] == g.PREC_SPLIT16F8 for t in tuned),
                         "tile_256": sum(t["tile_m"] == 256 for t in tuned),
                         "tile_128": sum(t["tile_m"] == 128 for t in tuned)},
            "unit": "s (host wall clock)", "line_search": "batched"}


def small_plain_cg_cpu(iters: int) -> dict:
    """The reference's side of small_plain_cg: `iters` PR+ CG iterations with the
    reference's line search on one host core through the reference's own compiled
    cpu.c (float; the CG control flow of gpair1/trunk/gpair.c:682-915 restated in
    the oracle; data built by the reference's getoifits.c, init_data and
    set_model). Runs in a worker thread beside the GPU blocks: the foreign calls
    release the GIL."""
    import numpy as np
    from oracle import oracle as O
    synth, _ = data_modules()
    _, oi = synth.make_workload_data("small")
    ref = _SampleProblem(reference_problem("small", oi))
    ev = O.RefEvaluator(ref)
    t0 = time.perf_counter()
    _, tr = ev.cg(np.maximum(ref.model, np.float32(1e-8)).astype(np.float32), iters, method=2)
    dt = time.perf_counter() - t0
    return {"s": dt, "cores": 1, "kind": "reference", "J": float(tr["J"][-1]),
            "criterion_evals": tr["criterion_evals"], "grad_evals": tr["grad_evals"],
            "note": "the reference's cpu.c criterion and gradients in float, one core"}


def small_plain_cg(iters: int, device: int, precisions, cpu=None) -> dict:
    """The plain method on the small workload (64x64, 0.1 mas/pixel, 900 V2, 600
    closure phases, MEM against a flat prior, alpha 1e-3): `iters` PR+ CG
    iterations with the reference's line search from the flat start on the GPU
    (one CUDA graph per run; device time and host wall clock, per precision
    path), beside `cpu` (small_plain_cg_cpu) when given."""
    import gpair_b200 as g
    p = g.workload_problem("small")
    img0 = p.start_image()
    names = {v: k for k, v in PRECISION_MODES.items()}
    out = {"workload": _describe("small", p), "iterations": iters, "method": "PR+, reference line search"}
    for prec in precisions:
        with g.Reconstructor(device) as r:
            r.set_problem(p)
            r.set_precision(prec)
            r.set_image(img0)
            r.cg(1, method=2)  # graph capture outside the timing
            r.set_image(img0)
            t0 = time.perf_counter()
            o = r.cg(iters, method=2)
            dt = time.perf_counter() - t0
            ms = r.last_run_stats()[0]
            out["gpu_" + names[prec]] = {"s": dt, "device_ms": ms, "J": o["J"], "criterion_evals": o["criterion_evals"],
                                         "grad_evals": o["grad_evals"]}
    if cpu is not None:
        out["cpu_reference"] = cpu
        for k, v in list(out.items()):
            if k.startswith("gpu_"):
                v["speedup_vs_cpu_reference"] = cpu["s"] / max(v["s"], 1e-12)
                v["rel_J_vs_cpu_reference"] = abs(v["J"] - cpu["J"]) / abs(cpu["J"])
    out["unit"] = "s (host wall clock of the whole run)"
    return out


def time_to_objective(n_problems: int, race_fr: bool = False, method: int = 2) -> dict:
    """CG time-to-objective on held-out problems of the warm-start workload (3/4
    at 64x64, 1/4 at 128x128): wall time until J <= J* (1 + 1e-4), J* = plain
    CG's converged objective (reference line search, 1000 iterations), for plain
    CG, the batched line search, the learned warm start (sequential fallback) and
    the warm start raced against a flat start in a second context."""
    import gpair_b200 as g
    from gpair_b200 import timetoobj as TT
    from gpair_b200.train_warmstart import SEED_HELD_OUT
    from gpair_b200.warmstart import WarmStartNet, training_case
    net = WarmStartNet.load()
    n64 = max(1, (3 * n_problems) // 4)
    rows = []
    flag = g.api.StopFlag()
    with g.Reconstructor(0) as rec, g.Reconstructor(0) as rec2, g.Reconstructor(0) as rec3:
        rec.set_precision(g.PREC_SPLIT16)
        for k in range(n_problems):
            p = training_case(SEED_HELD_OUT + k, 64 if k < n64 else 128).problem
            rows.append(TT.evaluate(rec, p, net, iters=1000, objective_from="plain", rec2=rec2, flag=flag,
                                    rec3=rec3 if race_fr else None, method=method))
    flag.close()
    out = TT.summarize(rows)
    out["unit"] = "s (sum of host wall clock over the problems)"
    out["workload"] = (f"{n_problems} held-out seeded problems ({n64} at 64x64 / 0.1 mas, {n_problems - n64} at "
                       "128x128 / 0.05 mas; 1-10 Gaussians/disks/points, 4-12 telescopes), tolerance 1e-4")
    out["direction"] = {2: "PR+ CG", 4: "projected L-BFGS"}[method] + " with the batched line search (batch, warm, race)"
    return out


def time_to_objective_workload(rec, p, iters: int, batch_iters: int, method: int = 2) -> dict:
    """Time-to-objective on the benchmark workload itself: plain CG (reference
    line search) for `iters` iterations sets J*, then plain CG, the batched line
    search from the flat prior and the batched line search from the learned
    warm start (the network applied at the workload's own size; the flat-prior
    run is the fallback) are each timed to J* (1 + 1e-4); then the warm start
    raced against the flat prior in a second context sharing a stop flag."""
    import gpair_b200 as g
    from gpair_b200 import timetoobj as TT
    from gpair_b200.warmstart import WarmStartNet
    net = WarmStartNet.load() if p.width % 8 == 0 else None
    flag = g.api.StopFlag() if net is not None else None
    rec2 = g.Reconstructor(rec.device) if net is not None else None
    try:
        if rec2 is not None:
            rec2.set_tc_pair(True)
        row = TT.evaluate(rec, p, net, iters=iters, batch_iters=batch_iters, objective_from="plain", method=method,
                          rec2=rec2, flag=flag)
    finally:
        if rec2 is not None:
            rec2.close()
        if flag is not None:
            flag.close()
    if net is not None:
        row["speedup_warm_vs_plain"] = row["plain_s"] / max(row["warm_s"], 1e-12)
        row["speedup_warm_vs_batch"] = row["batch_s"] / max(row["warm_s"], 1e-12)
        row["speedup_race_vs_plain"] = row["plain_s"] / max(row["race_s"], 1e-12)
        row["speedup_race_vs_batch"] = row["batch_s"] / max(row["race_s"], 1e-12)
    row["speedup_batch_vs_plain"] = row["plain_s"] / max(row["batch_s"], 1e-12)
    row["unit"] = "s (host wall clock)"
    row["note"] = f"J* = lowest J of {iters} plain PR+ iterations with the reference's line search"
    return row


def measure_plain(rec, p, args, flush, local, dist):
    """Timed plain CG iterations (device time, CUDA events inside the library),
    their per-stage times and the e2e leg through the public API."""
    import torch
    from gpair_b200.clocks import ClockSampler
    rec.cg(max(args.warmup, 1), method=2, resume=False, host_loop=int(args.host_loop),
           line_search=LS[args.line_search])  # untimed warm-up; builds the CG graph
    sampler = ClockSampler(local)
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.5)  # let the sampler take its first sample before the timed steps
    dev_ms, flops, launches, crit_evals, grad_evals = 0.0, 0.0, 0, 0, 0
    for k in range(args.steps):
        flush.fill_(float(k))  # 512 MiB write: L2 (126 MB) holds none of the inputs at step start
        torch.cuda.synchronize()
        out = rec.cg(1, method=2, resume=True, host_loop=int(args.host_loop), line_search=LS[args.line_search])
        ms, fl, nl = rec.last_run_stats()
        dev_ms += ms
        flops += fl
        launches += nl
        crit_evals += out["criterion_evals"]
        grad_evals += out["grad_evals"]
    torch.cuda.synchronize()
    if dist:
        torch.distributed.barrier()
    time.sleep(0.3)
    clocks = sampler.stop()

    # per-kernel times for the roofline: every stage of criterion + gradient
    # evaluations queued back to back on the library's stream and bracketed by
    # CUDA events (after an L2 flush), on the state the timed steps left
    flush.fill_(0.0)
    torch.cuda.synchronize()
    st = rec.time_stages(reps=min(args.steps, 10))
    crit_stages = ("prep", "forward_dft", "vis_data")
    stage_n = {k: (crit_evals if k in crit_stages else grad_evals) for k in st}
    stage_ms = {k: st[k] * stage_n[k] for k in st}

    # e2e: the same steps through the public API with host buffers
    img = rec.get_image()
    e2e_s, e2e_flops = 0.0, 0.0
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rec.set_image(img)  # H2D of the step's input image
        rec.cg(1, method=2, resume=True, host_loop=int(args.host_loop), line_search=LS[args.line_search])
        img = rec.get_image()  # D2H of the step's result
        e2e_s += time.perf_counter() - t0
        e2e_flops += rec.last_run_stats()[1]
    return {"dev_ms": dev_ms, "flops": flops, "launches": launches, "evals": crit_evals + grad_evals,
            "crit_evals": crit_evals, "grad_evals": grad_evals, "clocks": clocks, "stage_n": stage_n,
            "stage_ms": stage_ms, "e2e_s": e2e_s, "e2e_flops": e2e_flops, "img": img}


PRECISION_MODES = {"fp32": 0, "split16": 1, "split16f8": 4}
PRECISION_DTYPE = {
    "fp32": "fp32",
    "split16": "f16 hi+lo split operands (3 f16 products), fp32 accumulate",
    "split16f8": ("forward: f16 hi*hi + the two hi*lo cross terms as E4M3 products, one fp32 accumulator; "
                  "adjoint: f16 hi+lo split operands (3 f16 products); fp32 accumulate"),
}


def _executed_mult(precision, stage):
    """MMA work per algorithmic product in f16-rate units (1 for the CUDA-core path)."""
    if precision == "split16":
        return 3.0
    if precision == "split16f8":
        return 2.0 if stage.startswith("forward") else 3.0
    return 1.0


def roofline(p, m, precision, workload):
    """Roofline of the dominant stage (largest total time over the timed steps)."""
    hbm, tflops_peak, peak_kind = _peaks()
    stage_ms, stage_n = m["stage_ms"], m["stage_n"]
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    per_launch_ms = stage_ms[dom] / max(stage_n[dom], 1)
    if dom in ("forward_dft", "adjoint_dft"):
        work = p.dft_flops()
        achieved = work / (per_launch_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": tflops_peak, "unit": "TFLOP/s",
                "frac": achieved / tflops_peak, "work_per_launch": work,
                "work_note": "algorithmic FLOPs 4 N^2 nuv + 8 N nuv per launch (one image)"}
        mult = _executed_mult(precision, dom)  # MMA work per algorithmic product, in f16-rate units
        roof["executed_tflops"] = mult * achieved
        roof["executed_frac"] = mult * achieved / tflops_peak
        roof["executed_note"] = ("split16 issues 3 f16 MMAs (hi*hi, hi*lo, lo*hi) per algorithmic product; "
                                 "split16f8's forward 1 f16 MMA (hi*hi) and 2 E4M3 MMAs (the cross terms) at twice "
                                 "the f16 rate: 2 f16-rate units")
    else:
        bytes_per = {"prep": 8 * p.npix, "vis_data": 16 * p.npow + 60 * p.nbis,
                     "adj_weights": 8 * p.npow + 24 * p.nbis, "grad_finalize": 16 * p.npix}[dom]
        achieved = bytes_per / (per_launch_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "work_per_launch": bytes_per}
    roof["kernel"] = dom
    roof["peak_source"] = peak_kind
    roof["timing"] = ("per-stage CUDA events, stages queued back to back; stage totals = per-launch time x "
                      "the timed steps' criterion (prep, forward, vis_data) or gradient evaluations")
    roof["traffic"] = _traffic(f"{dom}@{workload}@{precision}")
    roof["stage_ms_per_launch"] = {k: stage_ms[k] / max(stage_n[k], 1) for k in stage_ms}
    roof["stage_share"] = {k: stage_ms[k] / max(sum(stage_ms.values()), 1e-12) for k in stage_ms}
    return roof


def batched_block(rec, p, args, flush, img, precision, workload):
    """The same CG iterations with the batched line search (8 trial images per
    tcgen05 forward launch), device-timed like the headline steps."""
    import torch
    import gpair_b200 as g
    hbm, tflops_peak, peak_kind = _peaks()
    bat_ms, bat_flops, bat_evals = 0.0, 0.0, 0
    rec.set_image(img)
    rec.cg(max(args.warmup, 1), method=2, resume=False, line_search=g.LS_BATCH, host_loop=int(args.host_loop))
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        out_b = rec.cg(1, method=2, resume=True, line_search=g.LS_BATCH, host_loop=int(args.host_loop))
        ms_b, fl_b, _ = rec.last_run_stats()
        bat_ms += ms_b
        bat_flops += fl_b
        bat_evals += out_b["criterion_evals"] + out_b["grad_evals"]
    flush.fill_(0.0)
    torch.cuda.synchronize()
    st_b = rec.time_batch_stages(reps=min(args.steps, 10))
    mult = _executed_mult(precision, "forward_dft")
    fb_ms = st_b["forward_dft_batch"]
    fb_ach = 8 * p.dft_flops() / (fb_ms * 1e-3) / 1e12
    return {"value": bat_flops / max(bat_ms * 1e-3, 1e-12) / 1e12, "unit": UNIT,
            "ms_per_step": bat_ms / max(args.steps, 1), "evaluations": bat_evals,
            "note": "CG iterations with 8 trial images per batched evaluation (rank 0, device time)",
            "roofline": {"bound": "tensor", "kernel": "forward_dft_batch (8 stacked trial images)",
                         "achieved": fb_ach, "peak": tflops_peak, "unit": "TFLOP/s", "frac": fb_ach / tflops_peak,
                         "executed_tflops": mult * fb_ach, "executed_frac": mult * fb_ach / tflops_peak,
                         "peak_source": peak_kind,
                         "traffic": _traffic(f"forward_dft_batch8@{workload}@{precision}"),
                         "stage_ms_per_launch": st_b,
                         "timing": "CUDA events around the three batched stages queued back to back"}}


def _describe(name, p):
    return f"{name}: {p.width}x{p.width} image, {p.npow} V2, {p.nbis} T3, nuv {p.nuv}"


def run_ours(args, rank, world, local):
    import torch
    import gpair_b200 as g
    from gpair_b200 import synth

    dist = world > 1
    if dist:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    # one independent replica per rank: same array and scene, own noise seed
    seeds = replica_seeds(rank)
    w, oi = synth.make_workload_data(args.workload, **seeds)
    p = g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha, modeltype=0, modelflux=w.prior_flux)
    prec = PRECISION_MODES[args.precision]
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    rec = g.Reconstructor(local)
    rec.set_problem(p)
    rec.set_precision(prec)
    rec.set_tc_pair(args.tc_pair)
    rec.set_stage_timing(True)
    rec.set_image(p.start_image())
    # autotuned adjoint split-K length (precision stays as requested)
    tune = rec.autotune(g.api.TUNE_SPLITS, reps=3)
    rec.set_image(p.start_image())

    m = measure_plain(rec, p, args, flush, local, dist)
    (max_ms, max_e2e), (tot_flops, tot_e2e_flops) = combine_over_ranks(
        [m["dev_ms"], m["e2e_s"]], [m["flops"], m["e2e_flops"]], f"cuda:{local}")
    # the same steps with three f16 products in the forward too, beside the headline
    split16 = None
    if args.precision == "split16f8":
        rec.set_precision(g.PREC_SPLIT16)
        rec.autotune(g.api.TUNE_SPLITS, reps=3)
        rec.set_image(p.start_image())
        m16 = measure_plain(rec, p, args, flush, local, dist)
        (ms16, e2e16), (fl16, e2efl16) = combine_over_ranks(
            [m16["dev_ms"], m16["e2e_s"]], [m16["flops"], m16["e2e_flops"]], f"cuda:{local}")
        split16 = {"value": fl16 / (ms16 * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms16 / args.steps,
                   "e2e": e2efl16 / e2e16 / 1e12, "dtype": PRECISION_DTYPE["split16"], "clocks": m16["clocks"],
                   "evaluations": m16["evals"]}
        rec.set_precision(prec)
        rec.autotune(g.api.TUNE_SPLITS, reps=3)
        rec.set_image(m["img"])

    if rank == 0:
        roof = roofline(p, m, args.precision, args.workload)
        value = tot_flops / (max_ms * 1e-3) / 1e12
        e2e = tot_e2e_flops / max_e2e / 1e12
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": PRECISION_DTYPE[args.precision],
                "data": "synthetic (seeded array, scene and noise; no public data set of this size)",
                "config": {"workload": _describe(args.workload, p),
                           "step": ("one PR+ CG iteration with strong-Wolfe line search (continuing)"
                                    if args.line_search == "wolfe" else
                                    "one PR+ CG iteration with the batched 8-trial line search (continuing)"),
                           "precision": args.precision, "evaluations": m["evals"],
                           "tensor_tiles": "CTA pairs (cta_group::2, 256x256)" if args.tc_pair else
                           "single CTAs (128x256)",
                           "criterion_evals": m["crit_evals"], "grad_evals": m["grad_evals"],
                           "flop_per_evaluation": p.dft_flops(),
                           "autotuned_adjoint_splits": tune["adjoint_splits"],
                           "l2": "flushed (512 MiB write) before every timed step, outside the timed region",
                           "parallelism": f"replicas x{world}", "seeds": seeds,
                           "cg_driver": "host loop" if args.host_loop else "one CUDA graph per step"},
                "gpu_launches": m["launches"], "clocks": m["clocks"], "roofline": roof,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 4 * p.npix,
                        "d2h_bytes_per_step": 4 * p.npix}}
        if split16 is not None:
            line["split16"] = split16
        if not args.no_batched:
            line["batched_line_search"] = batched_block(rec, p, args, flush, m["img"], args.precision, args.workload)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(reference_sample(args.workload, oi))
        if not args.no_time_to_objective and args.tto_workload_iters > 0:
            line["time_to_objective_workload"] = time_to_objective_workload(
                rec, p, args.tto_workload_iters, args.tto_workload_iters, args.tto_method)
    rec.close()
    del oi, p

    if rank == 0:
        # the reference's cpu.c on the small workload, in a worker thread beside the GPU blocks
        cpu_pool = cpu_small = None
        if args.small_iters > 0 and not args.no_cpu_baseline:
            import concurrent.futures
            cpu_pool = concurrent.futures.ThreadPoolExecutor(1)
            sys.stdout.flush()
            saved_fd, devnull_fd = os.dup(1), os.open(os.devnull, os.O_WRONLY)
            os.dup2(devnull_fd, 1)  # cpu.c's image2vis prints on every call
            cpu_small = cpu_pool.submit(small_plain_cg_cpu, args.small_iters)
        # the 256x256 precision workload beside the headline (context, same step)
        if args.workload != "precision" and not args.no_precision_256:
            p2 = g.workload_problem("precision", **seeds)
            with g.Reconstructor(local) as r2:
                r2.set_problem(p2)
                r2.set_precision(prec)
                r2.set_tc_pair(args.tc_pair)
                r2.set_stage_timing(True)
                r2.set_image(p2.start_image())
                r2.autotune(g.api.TUNE_SPLITS, reps=3)
                r2.set_image(p2.start_image())
                m2 = measure_plain(r2, p2, args, flush, local, False)
                blk = {"workload": _describe("precision", p2), "value": m2["flops"] / (m2["dev_ms"] * 1e-3) / 1e12,
                       "unit": UNIT, "ms_per_step": m2["dev_ms"] / args.steps, "evaluations": m2["evals"],
                       "gpu_launches": m2["launches"], "clocks": m2["clocks"],
                       "e2e": {"value": m2["e2e_flops"] / m2["e2e_s"] / 1e12, "unit": UNIT},
                       "roofline": roofline(p2, m2, args.precision, "precision")}
                if not args.no_batched:
                    blk["batched_line_search"] = batched_block(r2, p2, args, flush, m2["img"], args.precision,
                                                               "precision")
                line["precision_256"] = blk
        if not args.no_time_to_objective:
            line["time_to_objective"] = time_to_objective(args.tto_problems, race_fr=args.tto_race_fr,
                                                          method=args.tto_method)
        if args.instances > 0:
            line["many_instances"] = many_instances(args.instances, args.instance_iters, prec)
        if args.small_iters > 0:
            cpu = None
            if cpu_small is not None:
                try:
                    cpu = cpu_small.result()
                finally:
                    cpu_pool.shutdown()
                    os.dup2(saved_fd, 1)
                    os.close(saved_fd)
                    os.close(devnull_fd)
            line["small_plain_cg"] = small_plain_cg(args.small_iters, local, (g.PREC_FP32, prec), cpu)
        print(json.dumps(line), flush=True)
    if dist:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "precision", "small", "tiny"])
    ap.add_argument("--precision", default=os.environ.get("GPAIR_BENCH_PRECISION", "split16f8"),
                    choices=["fp32", "split16", "split16f8"],
                    help="split16f8 (default): f16 hi*hi + E4M3 cross terms in the forward, split-f16 adjoint; "
                         "every mode meets the 1e-5 bounds against the FP64 oracle (tests/)")
    ap.add_argument("--tc-pair", type=int, choices=[0, 1], default=1,
                    help="tensor-core contractions on CTA pairs (cta_group::2) instead of single CTAs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-time-to-objective", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched line-search block")
    ap.add_argument("--no-precision-256", action="store_true", help="skip the 256x256 context block")
    ap.add_argument("--instances", type=int, default=64, help="independent reconstructions run at once (0: skip)")
    ap.add_argument("--instance-iters", type=int, default=30)
    ap.add_argument("--small-iters", type=int, default=200,
                    help="plain CG iterations of the 64x64 workload on the GPU and the reference's cpu.c (0: skip)")
    ap.add_argument("--line-search", choices=["wolfe", "batch"], default="wolfe",
                    help="line search of the headline steps: the reference's (default) or the batched one")
    ap.add_argument("--tto-problems", type=int, default=16,
                    help="held-out warm-start problems timed for the time-to-objective block")
    ap.add_argument("--tto-workload-iters", type=int, default=60,
                    help="plain-CG iterations that set J* for the time-to-objective block on the benchmark "
                         "workload itself (0: skip)")
    ap.add_argument("--tto-method", type=int, choices=[2, 4], default=4,
                    help="direction of the batched / warm-start runs in the time-to-objective blocks: 2 PR+ CG, "
                         "4 projected L-BFGS")
    ap.add_argument("--tto-race-fr", action="store_true",
                    help="add a flat-start Fletcher-Reeves runner to the time-to-objective race")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the line search from the host instead of the CUDA graph (for profilers that do "
                         "not see kernels inside conditional graph nodes)")
    args = ap.parse_args()
    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
