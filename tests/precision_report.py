"""Precision report (test infrastructure): errors of the CUDA path against the
FP64 oracle, per quantity, for every precision mode the library builds.

    python tests/precision_report.py [--large] > report.md

Quantities, all on a random positive image (the flat prior x U(1, 3)):
  V        max |V - V64| (V normalised by the total flux), over every uv point
           (64^2, 256^2) or 256 random ones (1024^2)
  chi2     |chi2 - chi2_64| / chi2_64; chi2_64 from the FP64 visibilities
  grad     relative L2 error of the data gradient: the whole image (64^2,
           FP64 oracle gradient) or 24 random pixels (256^2, 1024^2), where
           the reference's direct per-pixel sum is evaluated in FP64 with the
           device's own visibilities and mock data
  entropy  |S - S64| / |S64|
"""
import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import gpair_b200 as g  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _mock_chi2(p, V):
    V = V.astype(np.complex128)
    mock = np.empty(p.npow + 2 * p.nbis)
    mock[:p.npow] = np.abs(V[:p.npow]) ** 2
    Vt = V[p.uvpnt]
    Vt = np.where(p.sign < 0, np.conj(Vt), Vt)
    t3 = Vt[:, 0] * Vt[:, 1] * Vt[:, 2] * p.phasor.astype(np.complex128)
    mock[p.npow::2] = t3.real
    mock[p.npow + 1::2] = t3.imag
    chi2 = float(np.sum(((mock - p.data.astype(np.float64)) * p.data_err.astype(np.float64)) ** 2))
    return mock, chi2


def _entropy64(img, model):
    img = img.astype(np.float64)
    m = model.astype(np.float64)
    ok = (img > 0) & (m > 0)
    return float(np.sum(np.where(ok, img - m - img * np.log(np.where(ok, img / m, 1.0)), -m)))


_PROBLEMS = {}


def measure(name, prec, nsel=None, npx=24, seed=5):
    if name not in _PROBLEMS:
        _PROBLEMS[name] = g.workload_problem(name)
    p = _PROBLEMS[name]
    rng = np.random.default_rng(seed)
    img = (p.start_image() * (1 + rng.uniform(0, 2, p.npix))).astype(np.float32)
    with g.Reconstructor(0) as rec:
        rec.set_problem(p)
        rec.set_precision(prec)
        rec.set_image(img)
        chi2, S = rec.criterion()
        V = rec.visibilities()
        rec.gradient()
        grad = rec.data_gradient().astype(np.float64)
        st = rec.time_stages(reps=10)  # CUDA events, stages back to back
    out = {"workload": name, "N": p.width, "nuv": p.nuv, "forward_ms": st["forward_dft"],
           "adjoint_ms": st["adjoint_dft"]}
    if p.width <= 64:
        e = O.evaluate64(p, img)
        out["V"] = float(np.abs(V - e["visi"]).max())
        out["chi2"] = abs(chi2 - e["chi2"]) / e["chi2"]
        out["grad"] = float(np.linalg.norm(grad - e["data_grad"]) / np.linalg.norm(e["data_grad"]))
        out["grad_on"] = "all pixels"
    else:
        sel = np.arange(p.nuv) if nsel is None else rng.choice(p.nuv, nsel, replace=False)
        V64 = O.visibilities_subset64(p, img, sel)
        out["V"] = float(np.abs(V[sel] - V64).max())
        out["V_on"] = "all uv" if nsel is None else f"{nsel} random uv"
        if nsel is None:
            _, chi2_64 = _mock_chi2(p, V64)
            out["chi2"] = abs(chi2 - chi2_64) / chi2_64
        mock_dev, _ = _mock_chi2(p, V)
        px = rng.integers(0, p.width, npx)
        py = rng.integers(0, p.width, npx)
        g64 = O.data_gradient_pixels64(p, img, V, mock_dev, px, py)
        gd = grad[py * p.width + px]
        out["grad"] = float(np.linalg.norm(gd - g64) / np.linalg.norm(g64))
        out["grad_on"] = f"{npx} random pixels"
    out["entropy"] = abs(S - _entropy64(img, p.model)) / abs(_entropy64(img, p.model))
    return out


MODES = ((g.PREC_FP32, "fp32 (CUDA cores)"), (g.PREC_SPLIT16, "split16 (3 f16 products)"),
         (g.PREC_SPLIT16F8, "split16f8 (forward: f16 hi*hi + 2 E4M3 cross products)"),
         (g.PREC_TF32, "tf32 (1 TF32 product)"), (g.PREC_TF32X3, "tf32x3 (3 TF32 products)"))


def main():
    from gpair_b200.clocks import ClockSampler

    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true", help="also the 1024^2 workload (tensor modes)")
    args = ap.parse_args()
    rows = []
    sampler = ClockSampler(0)
    sampler.start()
    for name in ("small", "precision"):
        for prec, pname in MODES:
            r = measure(name, prec)
            r["precision"] = pname
            rows.append(r)
    if args.large:
        for prec, pname in MODES[1:]:
            r = measure("large", prec, nsel=256)
            r["precision"] = pname
            rows.append(r)
    clocks = sampler.stop()
    print("| workload | precision | max abs V error | chi2 rel. error | data gradient rel. L2 error | "
          "entropy rel. error | forward | adjoint |")
    print("|---|---|---|---|---|---|---|---|")
    for r in rows:
        v_on = f" ({r['V_on']})" if "V_on" in r else ""
        chi = f"{r['chi2']:.2e}" if "chi2" in r else "(consistency only)"
        print(f"| {r['workload']} {r['N']}², nuv {r['nuv']} | {r['precision']} | {r['V']:.2e}{v_on} | {chi} | "
              f"{r['grad']:.2e} ({r['grad_on']}) | {r['entropy']:.1e} | {r['forward_ms'] * 1e3:.1f} µs | "
              f"{r['adjoint_ms'] * 1e3:.1f} µs |")
    print(f"\nSM clock during the run: median {clocks.get('sm_mhz')} MHz of max {clocks.get('sm_max_mhz')} MHz, "
          f"throttle reasons {clocks.get('reasons')} ({clocks.get('samples')} samples). Stage times: CUDA events "
          "around the stages queued back to back (gpair_time_stages, 10 repetitions).")


if __name__ == "__main__":
    main()
