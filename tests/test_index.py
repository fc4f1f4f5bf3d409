"""The product's OIFITS uv/triangle indexer against the reference's own get_oi_fits_data.

Bit-exact target: every output array (uv, uvpnt, sign, pow, ...) must be
identical to what gpair1/trunk/getoifits.c:65-357 produces, including the
order in which uv points are created and the first-match rule.
"""
import copy
import hashlib
import json
import os

import numpy as np
import pytest

import gpair_b200 as g
from gpair_b200 import synth
from gpair_b200.oifits import OIFits, T3Table, Vis2Table, WavelengthTable, read_oifits
from oracle import oracle as O

from conftest import reference_fixture_path

KEYS = ["pow", "powerr", "bisamp", "bisamperr", "bisphs", "bisphserr", "uv", "uvpnt", "sign"]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _same(ix, ref):
    assert (ix.npow, ix.nbis, ix.nuv) == (ref["npow"], ref["nbis"], ref["nuv"])
    for k in KEYS:
        a, b = getattr(ix, k), ref[k]
        assert a.shape == b.shape, k
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8)), k


def test_golden_small_index():
    """Committed output of the reference indexer (tests/golden/make_golden.py)."""
    w, oi = synth.make_workload_data("small", 1, 2, 3)
    ix = g.index_oifits(oi)
    gold = np.load(os.path.join(GOLDEN, "index_small.npz"))
    ref = {k: gold[k] for k in KEYS}
    ref.update(npow=len(gold["pow"]), nbis=len(gold["bisamp"]), nuv=len(gold["uv"]))
    _same(ix, ref)


@pytest.mark.parametrize("name,seeds", [("tiny", (1, 2, 3)), ("small", (4, 5, 6)), ("small", (7, 8, 9))])
def test_synthetic_matches_reference(name, seeds):
    w, oi = synth.make_workload_data(name, *seeds)
    _same(g.index_oifits(oi), O.ref_index(oi))


@pytest.mark.slow
def test_precision_workload_matches_reference():
    # 21,120 V2 + 70,400 triangles: ~20 s in the reference's linear matcher
    w, oi = synth.make_workload_data("precision", 1, 2, 3)
    _same(g.index_oifits(oi), O.ref_index(oi))


def _digest(ix):
    h = hashlib.sha256()
    for k in KEYS:
        h.update(np.ascontiguousarray(getattr(ix, k)).tobytes())
    return h.hexdigest()


@pytest.mark.skipif(reference_fixture_path() is None, reason="reference fixture not present")
def test_reference_oifits_fixture():
    fx = read_oifits(reference_fixture_path())
    with open(os.path.join(GOLDEN, "fixture_index.json")) as f:
        gold = json.load(f)
    for key, exp in gold.items():
        lo, hi = (float(x) for x in key.split("-", 1)) if not key.startswith("0.0-1e") else (0.0, 1e30)
        ix = g.index_oifits(fx, lo, hi)
        assert (ix.npow, ix.nbis, ix.nuv) == (exp["npow"], exp["nbis"], exp["nuv"])
        assert _digest(ix) == exp["sha256"]
        _same(ix, O.ref_index(fx, lo, hi))


def _tables(u1, v1, u2, v2, vis_u, vis_v, lam=(1.6e-6,), t3amp=None, flag_v=None, flag_t=None, target=1):
    lam = np.asarray(lam, np.float32)
    nw = len(lam)
    nv, nt = len(vis_u), len(u1)
    rng = np.random.default_rng(0)
    vis = Vis2Table("INS", np.full(nv, target, np.int32), np.asarray(vis_u, float), np.asarray(vis_v, float),
                    rng.uniform(0, 1, (nv, nw)), rng.uniform(0.01, 0.1, (nv, nw)),
                    np.zeros((nv, nw), np.uint8) if flag_v is None else flag_v)
    amp = rng.uniform(0, 1, (nt, nw)) if t3amp is None else t3amp
    t3 = T3Table("INS", np.full(nt, target, np.int32), np.asarray(u1, float), np.asarray(v1, float),
                 np.asarray(u2, float), np.asarray(v2, float), amp, rng.uniform(0.01, 0.1, (nt, nw)),
                 rng.uniform(-180, 180, (nt, nw)), np.ones((nt, nw)),
                 np.zeros((nt, nw), np.uint8) if flag_t is None else flag_t)
    return OIFits([WavelengthTable("INS", lam, np.full(nw, 1e-8, np.float32))], [vis], [t3], 1)


def test_edge_duplicates_conjugates_zero_u_nan_amplitudes():
    # V2 points: a duplicate pair, a u = 0 point, a point only matched by its conjugate
    vis_u = [10.0, 10.0, 0.0, -30.0, 55.0]
    vis_v = [5.0, 5.0, 7.0, 8.0, -2.0]
    u1 = [10.0, -10.0, 0.0, 30.0, 1e-30, 10.00001]
    v1 = [5.0, -5.0, 7.0, -8.0, 0.0, 5.0]
    u2 = [0.0, 30.0, -55.0, 0.0, 0.0, -10.0]
    v2 = [7.0, -8.0, 2.0, -7.0, 0.0, -5.0]
    amp = np.array([[0.5], [np.nan], [0.2], [np.nan], [0.1], [0.3]])
    oi = _tables(u1, v1, u2, v2, vis_u, vis_v, t3amp=amp)
    _same(g.index_oifits(oi), O.ref_index(oi))


def test_edge_flags_band_limits_and_targets():
    rng = np.random.default_rng(4)
    n = 40
    vu, vv = rng.uniform(-5e2, 5e2, n), rng.uniform(-5e2, 5e2, n)
    u1, v1 = vu[:20], vv[:20]
    u2, v2 = vu[20:], vv[20:]
    lam = (1.5e-6, 1.6e-6, 1.7e-6)
    fv = (rng.uniform(0, 1, (n, 3)) < 0.2).astype(np.uint8)
    ft = (rng.uniform(0, 1, (20, 3)) < 0.2).astype(np.uint8)
    oi = _tables(u1, v1, u2, v2, vu, vv, lam=lam, flag_v=fv, flag_t=ft)
    for lo, hi in ((0.0, 1e30), (1550.0, 1750.0), (1600.0, 1600.5), (2000.0, 3000.0)):
        _same(g.index_oifits(oi, lo, hi), O.ref_index(oi, lo, hi))
    # a table whose first record belongs to another target is skipped
    oi2 = _tables(u1, v1, u2, v2, vu, vv, lam=lam, target=7)
    _same(g.index_oifits(oi2, target_id=1), O.ref_index(oi2, target_id=1))


def test_edge_missing_wavelength_table_stops_reading():
    w, oi = synth.make_workload_data("tiny", 3, 4, 5)
    oi2 = copy.deepcopy(oi)
    extra = copy.deepcopy(oi.vis2[0])
    extra.insname = "OTHER"  # no OI_WAVELENGTH for this INSNAME
    oi2.vis2 = [oi.vis2[0], extra, copy.deepcopy(oi.vis2[0])]
    _same(g.index_oifits(oi2), O.ref_index(oi2))


def test_edge_empty_tables():
    w, oi = synth.make_workload_data("tiny", 3, 4, 5)
    oi2 = copy.deepcopy(oi)
    oi2.t3 = []
    _same(g.index_oifits(oi2), O.ref_index(oi2))
    oi3 = copy.deepcopy(oi)
    oi3.vis2 = []
    _same(g.index_oifits(oi3), O.ref_index(oi3))


def test_hash_candidates_cover_bucket_boundaries():
    # points straddling log2 bucket edges and the tiny-magnitude bucket
    base = np.array([2.0 ** k for k in range(-3, 20)] + [3 * 2.0 ** -62, 2.0 ** -60, 2.0 ** -61])
    vis_u = np.concatenate([base, base * (1 + 3e-5), -base * (1 - 3e-5)])
    vis_v = np.concatenate([base * 0.5, base * 0.5, -base * 0.5])
    u1 = base * (1 - 2e-5)
    v1 = base * 0.5
    u2 = -base * 0.25
    v2 = base * 0.1
    oi = _tables(u1, v1, u2, v2, vis_u, vis_v)
    _same(g.index_oifits(oi), O.ref_index(oi))


def test_fits_image_roundtrip(tmp_path):
    from gpair_b200.oifits import read_fits_image, write_fits_image
    rng = np.random.default_rng(0)
    img = rng.uniform(0, 1, (16, 24)).astype(np.float32)
    path = str(tmp_path / "img.fits")
    write_fits_image(path, img, {"PIXSCALE": 0.15, "ORIGIN": "test"})
    assert os.path.getsize(path) % 2880 == 0
    back, cards = read_fits_image(path)
    assert np.array_equal(back, img)
    assert cards["BITPIX"] == "-32" and float(cards["PIXSCALE"]) == 0.15


def test_cli_flags_mirror_the_reference_driver():
    from gpair_b200.reconstruct import build_parser
    a = build_parser().parse_args(["-d", "x.oifits", "-s", "0.2", "-w", "32", "-mt", "1", "-mw", "3", "-mf", "2",
                                   "-a", "0.001", "-wavmin", "1.5", "-wavmax", "2.0"])
    assert (a.data, a.pixellation, a.width, a.modeltype, a.modelwidth, a.modelflux) == ("x.oifits", 0.2, 32, 1, 3.0, 2.0)
    assert (a.alpha, a.minband, a.maxband) == (0.001, 1.5, 2.0)
    d = build_parser().parse_args([])
    # the reference's defaults (gpair1/trunk/gpair.c:78-85)
    assert (d.pixellation, d.modeltype, d.modelwidth, d.modelflux, d.alpha) == (0.15, 3, 5.0, 10.0, 1000.0)
