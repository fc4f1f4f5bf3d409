"""The CPU oracle pinned against the reference's own compiled code, plus known-answer tests.

The FP64 restatement (oracle/fp64) must agree with the reference's own
gpair1/trunk/cpu.c (compiled unchanged into oracle/_ref) to FP32 accuracy; the
exact-float setup replicas must agree bit for bit with the product's C setup
code and with the reference's set_model.
"""
import math

import numpy as np
import pytest

import gpair_b200 as g
from gpair_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available() and not __import__("os").path.exists(
    __import__("os").path.join(O.REFERENCE_TRUNK, "cpu.c")), reason="reference build unavailable")


@pytest.fixture(scope="module")
def small():
    w, oi = synth.make_workload_data("small", 11, 12, 13)
    return g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha)


@pytest.fixture(scope="module")
def tiny():
    w, oi = synth.make_workload_data("tiny", 21, 22, 23)
    return g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha)


def _rand_image(p, seed):
    rng = np.random.default_rng(seed)
    return (p.start_image() * (1 + rng.uniform(0, 2, p.npix))).astype(np.float32)


@pytest.mark.parametrize("which", ["tiny", "small"])
def test_fp64_oracle_matches_reference_cpu(which, request):
    p = request.getfixturevalue(which)
    img = _rand_image(p, 5)
    ev = O.RefEvaluator(p)
    chi2_ref = ev.chi2(img)
    e = O.evaluate64(p, img)
    assert abs(chi2_ref - e["chi2"]) / e["chi2"] < 2e-5
    # visibilities: FP32 reference vs FP64, relative to total flux (V is flux-normalised)
    assert np.abs(ev.visi[:p.nuv] - e["visi"]).max() < 2e-5
    assert np.allclose(ev.mock[:p.npow + 2 * p.nbis], e["mock"], rtol=1e-4, atol=1e-5)
    gref = ev.data_gradient(img)
    assert np.linalg.norm(gref - e["data_grad"]) / np.linalg.norm(e["data_grad"]) < 1e-4
    assert abs(ev.entropy(img) - e["entropy"]) <= 1e-4 * abs(e["entropy"]) + 1e-6
    eg_ref = ev.entropy_gradient(img)
    eg64 = O.entropy_gradient64(img, p.model)
    assert np.allclose(eg_ref, eg64, rtol=1e-5, atol=1e-6)


def test_entropy_gradient_keeps_previous_value_where_undefined(small):
    p = small
    img = _rand_image(p, 3)
    img[:10] = 0.0  # image <= 0: gradient keeps its previous value
    prev = np.full(p.npix, 7.0, np.float32)
    ev = O.RefEvaluator(p)
    got = ev.entropy_gradient(img, prev)
    assert np.all(got[:10] == 7.0)
    assert np.allclose(got[10:], -np.log(img[10:].astype(np.float64) / p.model[10:]), rtol=1e-6)


def test_init_data_replica_bit_exact(small):
    w, oi = synth.make_workload_data("small", 11, 12, 13)
    ix = g.index_oifits(oi)
    bisamperr = ix.bisamperr.copy()
    bisamperr[::7] = -1.0  # missing triple amplitudes -> extrapolated from V2
    bisamperr[::11] = 5e3
    ix.bisamperr = bisamperr
    d1, e1, p1, n1 = g.init_data(ix, 1)
    d2, e2, p2, n2 = O.init_data(ix.npow, ix.nbis, ix.pow, ix.powerr, ix.bisamp, bisamperr, ix.bisphs, ix.bisphserr,
                                 ix.uvpnt, 1)
    assert n1 == n2
    assert np.array_equal(d1.view(np.uint32), d2.view(np.uint32))
    assert np.array_equal(e1.view(np.uint32), e2.view(np.uint32))
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))


@pytest.mark.parametrize("do_extrapolation", [1, 0])
def test_init_data_bit_exact_with_reference(small, do_extrapolation):
    """The product's gpair_init_data against the reference's own init_data
    (gpair1/trunk/gpair.c:997-1066, compiled from its source): data packing,
    inverse errors, phasors and the ndof change, including missing triple
    amplitudes (extrapolated from V2), errors above 1e3, and triangles whose uv
    points carry no V2 point (no extrapolation: amplitude 1, error 1e99)."""
    if not __import__("os").path.exists(O.REF_MAIN_LIB):
        O.build()
    if not __import__("os").path.exists(O.REF_MAIN_LIB):
        pytest.skip("the reference's gpair.c is not built here")
    w, oi = synth.make_workload_data("small", 11, 12, 13)
    ix = g.index_oifits(oi)
    ix.bisamperr = ix.bisamperr.copy()
    ix.bisamperr[::7] = -1.0
    ix.bisamperr[::11] = 5e3
    ix.uvpnt = ix.uvpnt.copy()
    ix.uvpnt[3::13, 1] = ix.npow  # a uv point beyond the V2 points
    ix.uvpnt[5::17, 2] = ix.npow + 1
    d1, e1, p1, n1 = g.init_data(ix, do_extrapolation)
    d2, e2, p2, n2 = O.ref_init_data(ix.npow, ix.nbis, ix.pow, ix.powerr, ix.bisamp, ix.bisamperr, ix.bisphs,
                                     ix.bisphserr, ix.uvpnt, do_extrapolation)
    assert n1 == n2 and (n1 < 0) == bool(do_extrapolation)
    assert np.array_equal(d1.view(np.uint32), d2.view(np.uint32))
    assert np.array_equal(e1.view(np.uint32), e2.view(np.uint32))
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))


@pytest.mark.parametrize("modeltype,width,mw", [(0, 64, 0.0), (1, 64, 0.0), (2, 64, 1.0), (3, 256, 5.0),
                                                (4, 64, 2.0), (2, 33, 0.7)])
def test_set_model_bit_exact_with_reference(modeltype, width, mw):
    a = g.set_model(width, 0.1, modeltype, mw, 1.0)
    b = O.ref_set_model(width, 0.1, modeltype, mw, 1.0)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_dft_tables_bit_exact(small):
    p = small
    a = g.dft_tables(p.width, p.uv, p.pixellation)
    b = O.dft_tables_f32(p.width, p.uv, p.pixellation)
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    tx, ty, gx, gy = g.dft_tables(p.width, p.uv, p.pixellation, transposed=True)
    nuv, N = p.nuv, p.width
    assert np.array_equal(gx[:nuv * N].reshape(N, nuv), tx.reshape(nuv, N).T)
    assert np.all(gx[nuv * N:] == 0)


# ------------------------------------------------------------ known answers

def _single_problem(width=16, nuv=7, seed=0):
    rng = np.random.default_rng(seed)
    uv = np.zeros((nuv, 4), np.float32)
    uv[:, 0] = rng.uniform(0, 3e7, nuv)
    uv[:, 1] = rng.uniform(-3e7, 3e7, nuv)
    uv[:, 3] = 1.6e-6
    tri = np.array([[0, 1, 2], [1, 2, 3], [3, 4, 5], [6, 0, 5]], np.int64)
    sign = np.array([[1, -1, 1], [1, 1, -1], [-1, -1, 1], [1, 1, 1]], np.int16)
    nb = len(tri)
    data = np.abs(rng.normal(0.5, 0.2, nuv + 2 * nb)).astype(np.float32)
    data[nuv + 1::2] = 0
    err = rng.uniform(5, 20, nuv + 2 * nb).astype(np.float32)
    ph = np.exp(-1j * rng.uniform(-np.pi, np.pi, nb)).astype(np.complex64)
    model = np.full(width * width, 1.0 / (width * width), np.float32)
    return g.Problem(width, 0.2, uv, nuv, nb, data, err, ph, tri, sign, model, 1e-2)


def test_kat_point_source_at_origin_has_unit_visibility():
    p = _single_problem()
    img = np.zeros(p.npix)
    img[0] = 3.0
    e = O.evaluate64(p, img, want_grad=False)
    assert np.allclose(e["visi"], 1.0, atol=1e-14)
    assert np.allclose(e["mock"][:p.npow], 1.0, atol=1e-14)


def test_kat_shifted_delta_is_a_phase_ramp_with_reference_signs():
    p = _single_problem()
    x0, y0 = 3, 5
    img = np.zeros(p.npix)
    img[x0 + y0 * p.width] = 1.0
    e = O.evaluate64(p, img, want_grad=False)
    rp = (math.pi / 180) / 3.6e6 * p.pixellation
    u, v = p.uv[:, 0].astype(np.float64), p.uv[:, 1].astype(np.float64)
    expect = np.exp(2j * np.pi * rp * (u * x0 - v * y0))
    assert np.allclose(e["visi"], expect, atol=1e-12)


def _closed_triangle_problem(width, ntri, seed=0):
    """Triangles whose three uv points close (uv3 = -(uv1 + uv2)), folded to u >= 0 with signs."""
    rng = np.random.default_rng(seed)
    pts, tri, sign = [], [], []
    for t in range(ntri):
        a = rng.uniform(-3e7, 3e7, 2)
        b = rng.uniform(-3e7, 3e7, 2)
        row, srow = [], []
        for q in (a, b, -(a + b)):
            s = 1
            if q[0] < 0:
                q, s = -q, -1
            row.append(len(pts))
            srow.append(s)
            pts.append(q)
        tri.append(row)
        sign.append(srow)
    nuv = len(pts)
    uv = np.zeros((nuv, 4), np.float32)
    uv[:, :2] = np.array(pts)
    uv[:, 3] = 1.6e-6
    nd = nuv + 2 * ntri
    p = g.Problem(width, 0.2, uv, nuv, ntri, np.ones(nd, np.float32), np.ones(nd, np.float32),
                  np.ones(ntri, np.complex64), np.array(tri, np.int64), np.array(sign, np.int16),
                  np.full(width * width, 1.0 / width ** 2, np.float32))
    return p


def test_kat_closure_phase_of_point_symmetric_image_is_zero_or_pi():
    p = _closed_triangle_problem(17, 6)
    img = np.random.default_rng(4).uniform(0.1, 1, (17, 17))
    img = img + img[::-1, ::-1]  # symmetric about the centre pixel
    p.phasor[:] = 1.0
    e = O.evaluate64(p, img.ravel(), want_grad=False)
    t3 = e["mock"][p.npow::2] + 1j * e["mock"][p.npow + 1::2]
    # visibilities of a centro-symmetric image = real * phase ramp of the centre; closure removes the ramp
    # float32 uv storage leaves a closure error of ~1e-7 relative in u, v
    assert np.allclose(np.sin(np.angle(t3)), 0, atol=1e-6)


def test_kat_gradient_matches_finite_differences():
    p = _single_problem(width=8)
    rng = np.random.default_rng(9)
    img = rng.uniform(0.2, 1.0, p.npix)
    e = O.evaluate64(p, img)
    h = 1e-6
    for pix in (0, 9, 37, 63):
        ip, im = img.copy(), img.copy()
        ip[pix] += h
        im[pix] -= h
        fd = (O.evaluate64(p, ip, False)["chi2"] - O.evaluate64(p, im, False)["chi2"]) / (2 * h)
        assert abs(fd - e["data_grad"][pix]) <= 1e-6 * max(1.0, abs(fd))


def test_kat_entropy_gradient_is_minus_log_ratio():
    rng = np.random.default_rng(2)
    img = rng.uniform(0.01, 2, 100)
    m = rng.uniform(0.01, 2, 100).astype(np.float32)
    gr = O.entropy_gradient64(img, m)
    assert np.allclose(gr, -np.log(img / m.astype(np.float64)), rtol=0, atol=1e-14)


def test_fp64_cg_decreases_objective_and_matches_float_reference_cg(tiny):
    p = tiny
    img0 = p.start_image()
    _, tr64 = O.reconstruct64(p, img0, 12)
    assert tr64["J"][-1] < tr64["J"][0]
    assert np.all(np.diff(tr64["J"]) <= 1e-9 * np.abs(tr64["J"][:-1]))
    ev = O.RefEvaluator(p)
    _, tr32 = ev.cg(img0, 12)
    # the float CG over the reference's cpu.c follows the same decisions early on
    assert np.allclose(tr32["J"][:3], tr64["J"][:3], rtol=1e-4)
    assert np.allclose(tr32["step"][:3], tr64["step"][:3], rtol=1e-3)
    assert tr32["J"][-1] < tr32["J"][0]


def test_batched_line_search_oracle_descends_and_counts():
    """The FP64 restatement of the batched search: J never increases, each
    iteration costs one criterion of the current image plus whole batches of 8."""
    import gpair_b200 as g
    p = g.workload_problem("tiny", 21, 22, 23)
    iters = 5
    _, tr = O.reconstruct64(p, p.start_image(), iters, line_search=1)
    assert np.all(np.diff(tr["J"]) <= 0)
    assert tr["grad_evals"] == iters
    assert (tr["criterion_evals"] - iters) % 8 == 0
    assert np.all(tr["step"] > 0)


def test_projected_lbfgs_oracle_direction():
    """Method 4 (projected L-BFGS, a candidate for the device path): with the
    batched search its first iteration is PR+'s (both start from -g with the
    same search); with either search J never increases and the image stays on
    or above the positivity bound."""
    import gpair_b200 as g
    p = g.workload_problem("tiny", 21, 22, 23)
    iters = 30
    img_pr, tr_pr = O.reconstruct64(p, p.start_image(), iters, method=2, line_search=1)
    img_lb, tr_lb = O.reconstruct64(p, p.start_image(), iters, method=4, line_search=1)
    assert tr_lb["J"][0] == tr_pr["J"][0] and tr_lb["J"][1] == tr_pr["J"][1]
    assert tr_lb["step"][0] == tr_pr["step"][0]
    assert np.all(np.diff(tr_lb["J"]) <= 0) and tr_lb["J"][-1] < tr_lb["J"][0]
    assert tr_lb["grad_evals"] == iters and (tr_lb["criterion_evals"] - iters) % 8 == 0
    assert img_lb.min() >= 1e-8 * (1 - 1e-12)
    # a different direction from the second iteration on
    assert tr_lb["J"][-1] != tr_pr["J"][-1]
    # with the reference's search (curvature constant 0.9): Armijo steps, so J never increases
    img_w, tr_w = O.reconstruct64(p, p.start_image(), iters, method=4, line_search=0)
    assert np.all(np.diff(tr_w["J"]) <= 0) and tr_w["J"][-1] < tr_w["J"][0]
    assert img_w.min() >= 1e-8 * (1 - 1e-12) and tr_w["grad_evals"] >= iters
    with pytest.raises(ValueError):
        O.reconstruct64(p, p.start_image(), 2, method=5, line_search=1)


def _lbfgs_pairs(n, m, seed):
    """Pairs with positive curvature from a random SPD quadratic (y = A s)."""
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n)) / np.sqrt(n)
    A = B @ B.T + np.diag(rng.uniform(0.5, 2.0, n))
    S = rng.standard_normal((m, n))
    Y = S @ A.T
    return S, Y


@pytest.mark.parametrize("m", [0, 1, 3, 4, 7])
def test_lbfgs_compact_form_equals_two_loop(m):
    """The compact form (the formulation for a device path) gives the two-loop
    recursion's direction, with pixels on the bound held fixed. The search
    keeps the newest 4 pairs, so with 7 given the compact form gets those 4."""
    n = 300
    S, Y = _lbfgs_pairs(n, m, seed=m)
    rng = np.random.default_rng(100 + m)
    image = rng.uniform(0.1, 2.0, n)
    image[rng.choice(n, 40, replace=False)] = 1e-8
    g = rng.standard_normal(n)
    gamma = float(S[-1] @ Y[-1] / (Y[-1] @ Y[-1])) if m else 1.0
    d2 = O.lbfgs_direction64(S, Y, gamma, image, g)
    dc = O.lbfgs_direction_compact(S[-4:], Y[-4:], gamma, image, g)
    assert np.linalg.norm(dc - d2) <= 1e-10 * np.linalg.norm(d2)
    fixed = (image <= 1e-8 * 1.000001) & (g > 0)
    assert np.all(d2[fixed] == 0) and fixed.any()
    assert d2 @ g < 0  # a descent direction


def test_lbfgs_direction_satisfies_newest_secant_equation():
    """With no pixel on the bound, -d(g = y_newest) = H y_newest = s_newest."""
    n, m = 200, 5
    S, Y = _lbfgs_pairs(n, m, seed=7)
    image = np.ones(n)
    gamma = float(S[-1] @ Y[-1] / (Y[-1] @ Y[-1]))
    d = O.lbfgs_direction64(S, Y, gamma, image, Y[-1])
    assert np.allclose(-d, S[-1], rtol=0, atol=1e-9 * np.abs(S[-1]).max())


def test_l2_regularizer_restatement_matches_reference():
    rng = np.random.default_rng(4)
    N = 24
    img = rng.uniform(0, 2, N * N).astype(np.float32)
    model = rng.uniform(0.5, 1.5, N * N).astype(np.float32)
    model[::7] = 0.0  # pixels without prior are skipped
    S_ref, gsum_ref = O.ref_l2(N, img, model)
    assert abs(O.l2_entropy64(img, model) - S_ref) <= 1e-5 * abs(S_ref)
    assert abs(O.l2_entropy_gradient64(img, model).sum() - gsum_ref) <= 1e-5 * abs(gsum_ref)
