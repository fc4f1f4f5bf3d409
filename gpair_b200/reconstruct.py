"""Command-line reconstruction driver: OIFITS in, FITS image out.

    python -m gpair_b200.reconstruct -d data.oifits [-s 0.15] [-w 64] [-mt 3] [-mw 5] [-mf 10]
        [-m model.fits] [-i init.fits] [-a 1000] [-wavmin 0] [-wavmax 1e30]
        [--iterations 500] [--method 2] [--line-search wolfe|batch] [--precision split16|fp32]
        [--regularizer gs|l2] [--warm-start] [--out reconst.fits] [--log run.jsonl]
        [--checkpoint run.ck] [--resume run.ck] [--report-every 10] [--device 0]

The single-dash flags and their defaults are those of the reference's driver
(gpair1/trunk/gpair.c:78-148): data file, pixellation (mas), image width,
prior type / width / flux (gpair1/trunk/cpu.c:645-749), prior and initial
images from FITS files, entropy hyperparameter alpha, and the wavelength band.
The reference asks for the band and the target interactively; here they are
flags, and the first target is used. The reference writes `reconst.fits`
periodically (gpair1/trunk/gpair.c:698-703); this driver writes it at the end, and
writes a checkpoint of the full CG state every --report-every iterations when
--checkpoint is given. --log writes one JSON line per iteration: J, chi2,
chi2 / ndof, alpha S, S, step, beta, the evaluation counts and the wall time.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from typing import Optional

import numpy as np

from . import api
from .oifits import OIFits, read_fits_image, read_oifits, write_fits_image


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="python -m gpair_b200.reconstruct", description=__doc__.split("\n")[0])
    ap.add_argument("-d", dest="data", help="OIFITS data file")
    ap.add_argument("-s", dest="pixellation", type=float, default=0.15, help="mas per pixel")
    ap.add_argument("-w", dest="width", type=int, default=64, help="image width (pixels)")
    ap.add_argument("-mt", dest="modeltype", type=int, default=3, help="prior type 0-4")
    ap.add_argument("-mw", dest="modelwidth", type=float, default=5.0, help="prior width (mas)")
    ap.add_argument("-mf", dest="modelflux", type=float, default=10.0, help="prior total flux")
    ap.add_argument("-m", dest="modelfile", default="", help="prior image (FITS), replaces -mt/-mw/-mf")
    ap.add_argument("-i", dest="initfile", default="", help="initial image (FITS)")
    ap.add_argument("-a", dest="alpha", type=float, default=1000.0, help="entropy hyperparameter")
    ap.add_argument("-wavmin", dest="minband", type=float, default=0.0)
    ap.add_argument("-wavmax", dest="maxband", type=float, default=1e30)
    ap.add_argument("--iterations", type=int, default=500)
    ap.add_argument("--method", type=int, default=2, help="0 SD, 1 FR, 2 PR+, 3 HS+")
    ap.add_argument("--line-search", choices=["wolfe", "batch"], default="wolfe")
    ap.add_argument("--precision", choices=["split16", "split16f8", "fp32"], default="split16",
                    help="split16: three f16 products; split16f8: E4M3 cross terms in the forward; fp32: CUDA cores")
    ap.add_argument("--regularizer", choices=["gs", "l2"], default="gs")
    ap.add_argument("--warm-start", action="store_true", help="start from the learned warm start")
    ap.add_argument("--out", default="reconst.fits")
    ap.add_argument("--log", default=None, help="JSON lines, one per iteration")
    ap.add_argument("--checkpoint", default=None, help="checkpoint file written every --report-every iterations")
    ap.add_argument("--resume", default=None, help="checkpoint to continue from")
    ap.add_argument("--report-every", type=int, default=10)
    ap.add_argument("--device", type=int, default=0)
    return ap


def run(args, oi: Optional[OIFits] = None, quiet: bool = False) -> dict:
    """Reconstruct; `oi` replaces reading args.data (tests, in-memory callers)."""
    say = (lambda *a: None) if quiet else (lambda *a: print(*a, flush=True))
    if oi is None:
        if not args.data:
            raise SystemExit("no data file (-d)")
        oi = read_oifits(args.data)
    N = args.width
    p = api.problem_from_oifits(oi, N, args.pixellation, args.alpha, args.modeltype, args.modelwidth, args.modelflux,
                                args.minband, args.maxband)
    if args.modelfile:
        m, _ = read_fits_image(args.modelfile)
        if m.shape != (N, N):
            raise SystemExit(f"prior image is {m.shape}, expected {(N, N)}")
        p.model = m.ravel().astype(np.float32)
    start = p.start_image()
    if args.initfile:
        im, _ = read_fits_image(args.initfile)
        if im.shape != (N, N):
            raise SystemExit(f"initial image is {im.shape}, expected {(N, N)}")
        start = np.maximum(im.ravel(), np.float32(1e-8)).astype(np.float32)
    say(f"data: {p.npow} V2, {p.nbis} T3, {p.nuv} uv; image {N}x{N} at {args.pixellation} mas")
    ndof = p.npow + 2 * p.nbis
    ls = {"wolfe": api.LS_WOLFE, "batch": api.LS_BATCH}[args.line_search]
    log = open(args.log, "w") if args.log else None
    t0 = time.perf_counter()
    with api.Reconstructor(args.device) as rec:
        rec.set_problem(p)
        rec.set_precision({"split16": api.PREC_SPLIT16, "split16f8": api.PREC_SPLIT16F8,
                           "fp32": api.PREC_FP32}[args.precision])
        rec.set_regularizer({"gs": api.REG_GULL_SKILLING, "l2": api.REG_L2}[args.regularizer])
        resume = False
        if args.resume:
            rec.load_checkpoint(args.resume)
            resume = True
            say(f"resumed from {args.resume}")
        else:
            if args.warm_start and not args.initfile:
                from .warmstart import WarmStartNet, warm_start
                start = warm_start(WarmStartNet.load(device=args.device), rec, p)
            rec.set_image(start)
        done, evals_c, evals_g = 0, 0, 0
        last = {}
        while done < args.iterations:
            k = min(args.report_every, args.iterations - done)
            out = rec.cg(k, method=args.method, trace=True, resume=resume, line_search=ls)
            resume = True
            n = out["iterations"]
            evals_c += out["criterion_evals"]
            evals_g += out["grad_evals"]
            for j in range(n):
                J, chi2, S = out["trace_J"][j], out["trace_chi2"][j], out["trace_entropy"][j]
                last = {"iteration": done + j + 1, "J": J, "chi2": chi2, "chi2_ndof": chi2 / max(ndof, 1),
                        "alpha_S": args.alpha * S, "S": S, "step": out["trace_step"][j], "beta": out["trace_beta"][j]}
                if log:
                    log.write(json.dumps({**last, "criterion_evals": evals_c, "grad_evals": evals_g,
                                          "wall_s": time.perf_counter() - t0}) + "\n")
            done += n
            if last:
                say(f"it {last['iteration']:5d}  J {last['J']:.6g}  chi2/ndof {last['chi2_ndof']:.4g}  "
                    f"S {last['S']:.6g}  step {last['step']:.3g}")
            if args.checkpoint:
                rec.save_checkpoint(args.checkpoint, {"iteration": done})
            if n < k:  # stopped early (non-finite values)
                break
        img = rec.get_image().reshape(N, N)
    if log:
        log.close()
    write_fits_image(args.out, img, {"PIXSCALE": float(args.pixellation), "ALPHA": float(args.alpha),
                                     "ITERS": int(done), "CHI2": float(last.get("chi2", 0.0)),
                                     "ORIGIN": "gpair_b200"})
    say(f"wrote {args.out} after {done} iterations ({time.perf_counter() - t0:.2f} s)")
    return {"iterations": done, "final": last, "image": img}


def main(argv=None):
    args = build_parser().parse_args(argv)
    run(args)


if __name__ == "__main__":
    main(sys.argv[1:])
