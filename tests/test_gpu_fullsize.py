"""Parity at the full workload sizes, where the FP64 oracle cannot run the whole
problem: the CUDA path is checked on random subsets and through exact
consistency relations.

  visibilities   |V - V64| <= 1e-5 on 64 random uv points (FP64 DFT of the same image)
  data stage     mock data and chi2 recomputed in FP64 from the device's own
                 visibilities: chi2 within 1e-6 relative, mock within float rounding
  gradient       device data gradient on 24 random pixels against the reference's
                 direct per-pixel sum in FP64, evaluated with the device's
                 visibilities: relative L2 error <= 1e-5
  entropy        FP64 sums of FP32 per-pixel terms (tensor paths): 1e-6 relative
"""
import numpy as np
import pytest

import gpair_b200 as g
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _host_mock_chi2(p, V):
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


def _check(p, prec, seed=5, pair=True):
    rng = np.random.default_rng(seed)
    img = (p.start_image() * (1 + rng.uniform(0, 2, p.npix))).astype(np.float32)
    with g.Reconstructor(0) as rec:
        rec.set_problem(p)
        rec.set_precision(prec)
        rec.set_tc_pair(pair)
        rec.set_image(img)
        chi2, S = rec.criterion()
        V = rec.visibilities()
        mock = rec.mock()
        rec.gradient()
        grad = rec.data_gradient()
    sel = rng.choice(p.nuv, 64, replace=False)
    V64 = O.visibilities_subset64(p, img, sel)
    assert np.abs(V[sel] - V64).max() <= 1e-5
    mock64, chi2_host = _host_mock_chi2(p, V)
    assert abs(chi2 - chi2_host) <= 1e-6 * chi2_host
    assert np.allclose(mock, mock64, rtol=2e-6, atol=1e-6)
    assert abs(S - _entropy64(img, p.model)) <= (1e-12 if prec == g.PREC_FP32 else 1e-6) * max(1.0, abs(S))
    px = rng.integers(0, p.width, 24)
    py = rng.integers(0, p.width, 24)
    g64 = O.data_gradient_pixels64(p, img, V, mock64, px, py)
    gd = grad[py * p.width + px].astype(np.float64)
    assert np.linalg.norm(gd - g64) <= 1e-5 * np.linalg.norm(g64)


@pytest.fixture(scope="module")
def precision_problem():
    return g.workload_problem("precision")


@pytest.mark.parametrize("prec", [g.PREC_FP32, g.PREC_SPLIT16, g.PREC_TF32X3, g.PREC_SPLIT16F8])
def test_precision_workload_256(precision_problem, prec):
    _check(precision_problem, prec)


def test_precision_workload_256_single_ctas(precision_problem):
    _check(precision_problem, g.PREC_SPLIT16, pair=False)


@pytest.fixture(scope="module")
def large_problem():
    return g.workload_problem("large")


@pytest.mark.parametrize("pair,prec", [(False, g.PREC_SPLIT16), (True, g.PREC_SPLIT16), (True, g.PREC_SPLIT16F8)])
def test_large_workload_1024(large_problem, pair, prec):
    p = large_problem
    assert (p.width, p.npow, p.nbis) == (1024, 194560, 1167360)
    _check(p, prec, pair=pair)
