"""Regenerates the golden fixtures in tests/golden from the reference's own code.

Run here, where the reference sources are present (oracle/_ref is built from
them). The fixtures are outputs of the reference on seeded synthetic inputs:

  index_small.npz   get_oi_fits_data (gpair1/trunk/getoifits.c:65-357) on the
                    'small' synthetic tables (seeds 1, 2, 3): uv, uvpnt, sign, pow ...
  eval_tiny.npz     image2chi2 + compute_data_gradient (gpair1/trunk/cpu.c) on the
                    'tiny' problem at its start image and at a perturbed image
  fixture_index.json  sha256 of the reference's indexer output on the reference's
                    OIFITS fixture (no data from the fixture is stored)

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import gpair_b200 as g  # noqa: E402
from gpair_b200 import synth  # noqa: E402
from gpair_b200.oifits import read_oifits  # noqa: E402
from oracle import oracle as O  # noqa: E402

FIXTURE = os.path.join(O.REFERENCE_TRUNK, "2004contest1.oifits")
KEYS = ["pow", "powerr", "bisamp", "bisamperr", "bisphs", "bisphserr", "uv", "uvpnt", "sign"]


def index_digest(d):
    h = hashlib.sha256()
    for k in KEYS:
        h.update(np.ascontiguousarray(d[k]).tobytes())
    return h.hexdigest()


def main():
    w, oi = synth.make_workload_data("small", 1, 2, 3)
    r = O.ref_index(oi)
    np.savez_compressed(os.path.join(HERE, "index_small.npz"), **{k: r[k] for k in KEYS})

    w, oi = synth.make_workload_data("tiny", 21, 22, 23)
    p = g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha)
    ev = O.RefEvaluator(p)
    img0 = p.start_image()
    img1 = (img0 * (1 + np.random.default_rng(5).uniform(0, 2, p.npix))).astype(np.float32)
    out = {}
    for tag, img in (("start", img0), ("perturbed", img1)):
        out[f"{tag}_image"] = img
        out[f"{tag}_chi2"] = np.float32(ev.chi2(img))
        out[f"{tag}_visi"] = ev.visi[:p.nuv].copy()
        out[f"{tag}_mock"] = ev.mock[:p.npow + 2 * p.nbis].copy()
        out[f"{tag}_grad"] = ev.data_gradient(img)
        out[f"{tag}_entropy"] = np.float32(ev.entropy(img))
    np.savez_compressed(os.path.join(HERE, "eval_tiny.npz"), **out)

    if os.path.exists(FIXTURE):
        fx = read_oifits(FIXTURE)
        res = {}
        for lo, hi in ((0.0, 1e30), (600.0, 800.0)):
            d = O.ref_index(fx, lo, hi)
            res[f"{lo}-{hi}"] = {"npow": d["npow"], "nbis": d["nbis"], "nuv": d["nuv"], "sha256": index_digest(d)}
        with open(os.path.join(HERE, "fixture_index.json"), "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
