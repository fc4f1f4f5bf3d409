"""CPU oracle of the reconstruction path -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product (gpair_b200) never imports it.

Two native libraries, both built by oracle/Makefile:
* lib/liboracle_fp64.so -- FP64 restatement of the reference's math and CG
  (oracle/fp64/oracle_fp64.c), plus exact-float replicas of its setup code;
* _ref/libgpair_ref.so  -- the reference's own gpair1/trunk/cpu.c and
  gpair1/trunk/getoifits.c compiled unchanged, with an in-memory cfitsio shim
  (oracle/shim), used to pin the restatement and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's trunk sources, read in place (the one place this path is set;
# oracle/Makefile's REF has the same default)
REFERENCE_TRUNK = os.environ.get("GPAIR_REFERENCE_TRUNK", "/root/reference/gpair1/trunk")
FP64_LIB = os.path.join(HERE, "lib", "liboracle_fp64.so")
REF_LIB = os.path.join(HERE, "_ref", "libgpair_ref.so")
REF_MAIN_LIB = os.path.join(HERE, "_ref", "libgpair_ref_main.so")

_fp64 = None
_ref = None
_ref_main = None


def build():
    """Build the oracle libraries (reference part only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_TRUNK}"], check=True)


def _p(a):
    return None if a is None else a.ctypes.data


def fp64() -> C.CDLL:
    global _fp64
    if _fp64 is None:
        if not os.path.exists(FP64_LIB):
            build()
        L = C.CDLL(FP64_LIB)
        vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        L.o_init_data.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.o_dft_tables_f32.argtypes = [i, i, vp, f, vp, vp]
        L.o64_image2vis.argtypes = [i, i, vp, vp, f, vp]
        L.o64_vis2data.argtypes = [i, i, vp, vp, vp, vp, vp]
        L.o64_data2chi2.argtypes = [i, vp, vp, vp]
        L.o64_data2chi2.restype = d
        L.o64_entropy.argtypes = [i, vp, vp]
        L.o64_entropy.restype = d
        L.o64_entropy_gradient.argtypes = [i, vp, vp, vp]
        L.o64_data_gradient.argtypes = [i, i, i, vp, vp, f, vp, vp, vp, vp, vp, vp, vp, vp]
        L.o64_evaluate.argtypes = [i, i, i, i, vp, f, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(d), vp]
        L.o64_evaluate.restype = d
        L.o64_reconstruct.argtypes = [i, i, i, i, vp, f, vp, vp, vp, vp, vp, vp, d, i, i, vp, C.POINTER(i),
                                      C.POINTER(i), vp, vp, vp, vp, vp, i, d]
        L.o32_ref_cg_run.argtypes = [vp, i, i, i, vp, f, i, i, vp, vp, vp, vp, vp, C.POINTER(i), C.POINTER(i), vp, vp,
                                     vp, vp, vp]
        L.o_set_threads.argtypes = [i]
        L.o64_lbfgs_direction.argtypes = [i, i, vp, vp, d, vp, vp, d, vp]
        _fp64 = L
    return _fp64


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


class RefProblem(C.Structure):
    _fields_ = [("image_width", C.c_int), ("nuv", C.c_int), ("npow", C.c_int), ("nbis", C.c_int),
                ("data", C.c_void_p), ("data_err", C.c_void_p), ("phasor", C.c_void_p), ("uvpnt", C.c_void_p),
                ("sign", C.c_void_p), ("dft_x", C.c_void_p), ("dft_y", C.c_void_p)]


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not ref_available():
            build()
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB} not built (reference sources unavailable)")
        L = C.CDLL(REF_LIB)
        vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        L.oracle_shim_reset.argtypes = [i]
        L.oracle_shim_add_wavelength.argtypes = [C.c_char_p, i, vp, vp]
        L.oracle_shim_add_vis2.argtypes = [C.c_char_p, C.c_long, i, vp, vp, vp, vp, vp, vp]
        L.oracle_shim_add_t3.argtypes = [C.c_char_p, C.c_long, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.oracle_ref_get_oi_fits_data.argtypes = [i, f, f, C.c_long, C.c_long, C.POINTER(i), C.POINTER(i),
                                                  C.POINTER(i), i]
        L.oracle_ref_copy_oi_data.argtypes = [vp] * 9
        L.oracle_ref_image2chi2.argtypes = [C.POINTER(RefProblem), vp, vp, vp, i]
        L.oracle_ref_image2chi2.restype = f
        L.oracle_ref_data_gradient.argtypes = [C.POINTER(RefProblem), vp, vp, vp, vp]
        L.oracle_ref_entropy.argtypes = [i, vp, vp]
        L.oracle_ref_entropy.restype = f
        L.oracle_ref_entropy_gradient.argtypes = [i, vp, vp, vp]
        L.oracle_ref_set_model.argtypes = [i, f, i, f, f, vp, i]
        _ref = L
    return _ref


# ------------------------------------------------------------- indexing

def ref_index(oi, minband: float = 0.0, maxband: float = 1e30, target_id: Optional[int] = None):
    """Run the reference's get_oi_fits_data over OIFITS tables (gpair_b200.oifits.OIFits)."""
    L = ref()
    keep = []

    def a(x, dt):
        arr = np.ascontiguousarray(x, dtype=dt)
        keep.append(arr)
        return _p(arr)

    L.oracle_shim_reset(oi.target_id)
    for w in oi.wavelengths:
        L.oracle_shim_add_wavelength(w.insname.encode(), len(w.eff_wave), a(w.eff_wave, np.float32),
                                     a(w.eff_band, np.float32))
    for t in oi.vis2:
        L.oracle_shim_add_vis2(t.insname.encode(), len(t.ucoord), t.nwave, a(t.target_id, np.int32),
                               a(t.vis2data, np.float64), a(t.vis2err, np.float64), a(t.ucoord, np.float64),
                               a(t.vcoord, np.float64), a(t.flag, np.uint8))
    for t in oi.t3:
        L.oracle_shim_add_t3(t.insname.encode(), len(t.u1coord), t.nwave, a(t.target_id, np.int32),
                             a(t.t3amp, np.float64), a(t.t3amperr, np.float64), a(t.t3phi, np.float64),
                             a(t.t3phierr, np.float64), a(t.u1coord, np.float64), a(t.v1coord, np.float64),
                             a(t.u2coord, np.float64), a(t.v2coord, np.float64), a(t.flag, np.uint8))
    npow, nbis, nuv = C.c_int(), C.c_int(), C.c_int()
    tid = oi.target_id if target_id is None else target_id
    rc = L.oracle_ref_get_oi_fits_data(tid, minband, maxband, oi.num_vis2, oi.num_t3, C.byref(npow), C.byref(nbis),
                                       C.byref(nuv), 1)
    if rc:
        raise RuntimeError(f"reference get_oi_fits_data status {rc}")
    n, b, u = npow.value, nbis.value, nuv.value
    out = dict(npow=n, nbis=b, nuv=u, pow=np.zeros(n, np.float32), powerr=np.zeros(n, np.float32),
               bisamp=np.zeros(b, np.float32), bisamperr=np.zeros(b, np.float32), bisphs=np.zeros(b, np.float32),
               bisphserr=np.zeros(b, np.float32), uv=np.zeros((u, 4), np.float32), uvpnt=np.zeros((b, 3), np.int64),
               sign=np.zeros((b, 3), np.int16))
    L.oracle_ref_copy_oi_data(*[_p(out[k]) for k in ("pow", "powerr", "bisamp", "bisamperr", "bisphs", "bisphserr",
                                                     "uv", "uvpnt", "sign")])
    return out


def ref_init_data(npow, nbis, pow_, powerr, bisamp, bisamperr, bisphs, bisphserr, uvpnt, do_extrapolation=1):
    """The reference's own init_data (gpair1/trunk/gpair.c:997-1066, compiled with
    main renamed into oracle/_ref/libgpair_ref_main.so). Returns data, data_err,
    phasor (complex64) and the change of its global ndof."""
    global _ref_main
    if _ref_main is None:
        if not os.path.exists(REF_MAIN_LIB):
            build()
        if not os.path.exists(REF_MAIN_LIB):
            raise FileNotFoundError(f"{REF_MAIN_LIB} not built (reference sources unavailable)")
        L = C.CDLL(REF_MAIN_LIB)
        vp, i = C.c_void_p, C.c_int
        L.oracle_ref_init_data.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.oracle_ref_init_data.restype = i
        _ref_main = L
    nd = npow + 2 * nbis
    data = np.zeros(max(nd, 1), np.float32)
    err = np.zeros(max(nd, 1), np.float32)
    ph = np.zeros(max(nbis, 1), np.complex64)
    f32 = [np.ascontiguousarray(x, np.float32) for x in (pow_, powerr, bisamp, bisamperr, bisphs, bisphserr)]
    uv = np.ascontiguousarray(np.asarray(uvpnt, np.int64).reshape(-1, 3))
    delta = _ref_main.oracle_ref_init_data(do_extrapolation, npow, nbis, *[_p(x) for x in f32], _p(uv), _p(data),
                                           _p(err), _p(ph))
    return data[:nd], err[:nd], ph[:nbis], int(delta)


# ----------------------------------------------------------- setup replicas

def init_data(npow, nbis, pow_, powerr, bisamp, bisamperr, bisphs, bisphserr, uvpnt, do_extrapolation=1):
    L = fp64()
    nd = npow + 2 * nbis
    data = np.zeros(max(nd, 1), np.float32)
    err = np.zeros(max(nd, 1), np.float32)
    ph = np.zeros(max(nbis, 1), np.complex64)
    ba, be = np.array(bisamp, np.float32), np.array(bisamperr, np.float32)
    uvpnt = np.ascontiguousarray(uvpnt, np.int64)
    args = [np.ascontiguousarray(x, np.float32) for x in (pow_, powerr)]
    args2 = [np.ascontiguousarray(x, np.float32) for x in (bisphs, bisphserr)]
    delta = L.o_init_data(do_extrapolation, npow, nbis, _p(args[0]), _p(args[1]), _p(ba), _p(be), _p(args2[0]),
                          _p(args2[1]), _p(uvpnt), _p(data), _p(err), _p(ph))
    return data[:nd], err[:nd], ph[:nbis], int(delta)


def dft_tables_f32(width, uv, pix):
    uv = np.ascontiguousarray(uv, np.float32)
    nuv = uv.shape[0]
    tx = np.zeros(nuv * width, np.complex64)
    ty = np.zeros(nuv * width, np.complex64)
    fp64().o_dft_tables_f32(width, nuv, _p(uv), pix, _p(tx), _p(ty))
    return tx, ty


def ref_set_model(width, pix, modeltype, modelwidth, modelflux):
    m = np.zeros(width * width, np.float32)
    ref().oracle_ref_set_model(width, pix, modeltype, modelwidth, modelflux, _p(m), 1)
    return m


# -------------------------------------------------------------- FP64 math

def evaluate64(p, image, want_grad=True, threads: int = 8):
    """FP64 chi2, entropy, visibilities, mock and data gradient of `image` for a gpair_b200.Problem."""
    L = fp64()
    L.o_set_threads(threads)
    img = np.ascontiguousarray(image, np.float64)
    uv = np.ascontiguousarray(p.uv, np.float32)
    visi = np.zeros(max(p.nuv, 1), np.complex128)
    mock = np.zeros(max(p.npow + 2 * p.nbis, 1), np.float64)
    grad = np.zeros(p.npix, np.float64) if want_grad else None
    S = C.c_double()
    keep = [np.ascontiguousarray(x) for x in (p.data.astype(np.float32), p.data_err.astype(np.float32),
                                              p.phasor.astype(np.complex64), p.uvpnt.astype(np.int64),
                                              p.sign.astype(np.int16), p.model.astype(np.float32))]
    chi2 = L.o64_evaluate(p.width, p.nuv, p.npow, p.nbis, _p(uv), p.pixellation, _p(keep[0]), _p(keep[1]),
                          _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]), _p(img), _p(visi), _p(mock),
                          C.byref(S), _p(grad))
    return dict(chi2=chi2, entropy=S.value, visi=visi[:p.nuv], mock=mock[:p.npow + 2 * p.nbis], data_grad=grad)


def entropy_gradient64(image, model, prev=None):
    g = np.zeros(len(image), np.float64) if prev is None else np.array(prev, np.float64)
    img = np.ascontiguousarray(image, np.float64)
    m = np.ascontiguousarray(model, np.float32)
    fp64().o64_entropy_gradient(len(img), _p(img), _p(m), _p(g))
    return g


def reconstruct64(p, image, iterations, method=2, threads: int = 8, line_search: int = 0,
                  batch_step_max: float = 1e12):
    """FP64 CG from `image`; returns (image, trace dict). line_search 0: the
    reference's GPU-path control flow; 1: the batched 8-trial search. method:
    0 SD, 1 FR, 2 PR+, 3 HS+ (the reference's beta rules); 4 projected L-BFGS
    with 4 pairs, with either search (with the reference's search it uses the
    curvature constant c2 = 0.9 instead of 0.1; a candidate direction for the
    device path, not in the library yet)."""
    if line_search not in (0, 1):
        raise ValueError(f"line_search must be 0 (reference) or 1 (batched), got {line_search}")
    if method not in (0, 1, 2, 3, 4):
        raise ValueError(f"method must be 0-4, got {method}")
    L = fp64()
    L.o_set_threads(threads)
    img = np.ascontiguousarray(image, np.float64).copy()
    uv = np.ascontiguousarray(p.uv, np.float32)
    tr = [np.zeros(iterations, np.float64) for _ in range(5)]
    ce, ge = C.c_int(), C.c_int()
    keep = [np.ascontiguousarray(x) for x in (p.data.astype(np.float32), p.data_err.astype(np.float32),
                                              p.phasor.astype(np.complex64), p.uvpnt.astype(np.int64),
                                              p.sign.astype(np.int16), p.model.astype(np.float32))]
    rc = L.o64_reconstruct(p.width, p.nuv, p.npow, p.nbis, _p(uv), p.pixellation, _p(keep[0]), _p(keep[1]),
                           _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]), p.alpha, method, iterations, _p(img),
                           C.byref(ce), C.byref(ge), *[_p(t) for t in tr], C.c_int(line_search),
                           C.c_double(batch_step_max))
    if rc:
        raise RuntimeError("o64_reconstruct failed")
    return img, dict(criterion_evals=ce.value, grad_evals=ge.value, J=tr[0], chi2=tr[1], entropy=tr[2], step=tr[3],
                     beta=tr[4])


# ------------------------------------------- the reference's own cpu.c

class RefEvaluator:
    """The reference's compiled cpu.c on one problem (float, CPU DFT tables)."""

    def __init__(self, p, dft_x=None, dft_y=None):
        L = ref()
        self.p = p
        if dft_x is None:
            dft_x, dft_y = dft_tables_f32(p.width, p.uv, p.pixellation)
        self._keep = [np.ascontiguousarray(p.data, np.float32), np.ascontiguousarray(p.data_err, np.float32),
                      np.ascontiguousarray(p.phasor, np.complex64), np.ascontiguousarray(p.uvpnt, np.int64),
                      np.ascontiguousarray(p.sign, np.int16), np.ascontiguousarray(dft_x, np.complex64),
                      np.ascontiguousarray(dft_y, np.complex64)]
        k = self._keep
        self.prob = RefProblem(p.width, p.nuv, p.npow, p.nbis, _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]),
                               _p(k[5]), _p(k[6]))
        self.visi = np.zeros(max(p.nuv, 1), np.complex64)
        self.mock = np.zeros(max(p.npow + 2 * p.nbis, 1), np.float32)
        self.L = L

    def chi2(self, image):
        img = np.ascontiguousarray(image, np.float32).copy()
        return float(self.L.oracle_ref_image2chi2(C.byref(self.prob), _p(img), _p(self.visi), _p(self.mock), 1))

    def data_gradient(self, image):
        img = np.ascontiguousarray(image, np.float32).copy()
        g = np.zeros(self.p.npix, np.float32)
        self.L.oracle_ref_data_gradient(C.byref(self.prob), _p(img), _p(self.visi), _p(self.mock), _p(g))
        return g

    def entropy(self, image):
        img = np.ascontiguousarray(image, np.float32).copy()
        m = np.ascontiguousarray(self.p.model, np.float32)
        return float(self.L.oracle_ref_entropy(self.p.width, _p(img), _p(m)))

    def entropy_gradient(self, image, prev=None):
        img = np.ascontiguousarray(image, np.float32).copy()
        m = np.ascontiguousarray(self.p.model, np.float32)
        g = np.zeros(self.p.npix, np.float32) if prev is None else np.array(prev, np.float32)
        self.L.oracle_ref_entropy_gradient(self.p.width, _p(img), _p(m), _p(g))
        return g

    def cg(self, image, iterations, method=2):
        """Float CG (reference GPU-path control flow) over the reference's cpu.c. Returns (image, trace)."""
        F = fp64()
        img = np.ascontiguousarray(image, np.float32).copy()
        m = np.ascontiguousarray(self.p.model, np.float32).copy()
        tr = [np.zeros(iterations, np.float32) for _ in range(5)]
        ce, ge = C.c_int(), C.c_int()
        fn = lambda name: C.cast(getattr(self.L, name), C.c_void_p)  # noqa: E731
        rc = F.o32_ref_cg_run(C.addressof(self.prob), self.p.width, self.p.nuv, self.p.npow + 2 * self.p.nbis, _p(m),
                              self.p.alpha, method, iterations, _p(img), fn("oracle_ref_image2chi2"),
                              fn("oracle_ref_data_gradient"), fn("oracle_ref_entropy"),
                              fn("oracle_ref_entropy_gradient"), C.byref(ce), C.byref(ge), *[_p(t) for t in tr])
        if rc:
            raise RuntimeError("o32_ref_cg_run failed")
        return img, dict(criterion_evals=ce.value, grad_evals=ge.value, J=tr[0], chi2=tr[1], entropy=tr[2],
                         step=tr[3], beta=tr[4])


def visibilities_subset64(p, image, sel):
    """FP64 visibilities of `image` at uv indices `sel` (for checks at full problem size)."""
    L = fp64()
    L.o64_image2vis_subset.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    img = np.ascontiguousarray(image, np.float64)
    uv = np.ascontiguousarray(p.uv, np.float32)
    sel = np.ascontiguousarray(sel, np.int32)
    out = np.zeros(len(sel), np.complex128)
    L.o64_image2vis_subset(p.width, _p(img), _p(uv), p.pixellation, len(sel), _p(sel), _p(out))
    return out


def data_gradient_pixels64(p, image, visi, mock, px, py):
    """FP64 direct gradient (reference per-pixel sum) at pixels (px, py), given visibilities and mock data."""
    L = fp64()
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    L.o64_data_gradient_pixels.argtypes = [i, i, i, i, vp, vp, f, vp, vp, vp, vp, vp, vp, vp, i, vp, vp, vp]
    img = np.ascontiguousarray(image, np.float64)
    keep = [np.ascontiguousarray(x) for x in (p.uv.astype(np.float32), p.data.astype(np.float32),
                                              p.data_err.astype(np.float32), p.phasor.astype(np.complex64),
                                              p.uvpnt.astype(np.int64), p.sign.astype(np.int16))]
    v = np.ascontiguousarray(visi, np.complex128)
    m = np.ascontiguousarray(mock, np.float64)
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    out = np.zeros(len(px), np.float64)
    L.o64_data_gradient_pixels(p.width, p.npow, p.nbis, p.nuv, _p(img), _p(keep[0]), p.pixellation, _p(keep[1]),
                               _p(keep[2]), _p(keep[3]), _p(keep[4]), _p(keep[5]), _p(v), _p(m), len(px), _p(px),
                               _p(py), _p(out))
    return out


# ------------------------------------------------------------- regularisers

def l2_entropy64(image, model):
    """FP64 L2 regulariser, gpair1/trunk/cpu.c:508-521: sum over m > 0 of -I^2 / (2m)."""
    I = np.asarray(image, np.float64)
    m = np.asarray(model, np.float64)
    ok = m > 0
    return float(np.sum(np.where(ok, -I * I / (2.0 * np.where(ok, m, 1.0)), 0.0)))


def l2_entropy_gradient64(image, model):
    """Per-pixel gradient of l2_entropy64: -I/m where m > 0, else 0. The reference's
    L2_entropy_gradient (gpair1/trunk/cpu.c:523-534) returns the sum of this field."""
    I = np.asarray(image, np.float64)
    m = np.asarray(model, np.float64)
    ok = m > 0
    return np.where(ok, -I / np.where(ok, m, 1.0), 0.0)


def ref_l2(width, image, model):
    """The reference's compiled L2_entropy and L2_entropy_gradient (a scalar sum)."""
    L = ref()
    for name in ("L2_entropy", "L2_entropy_gradient"):
        getattr(L, name).restype = C.c_float
        getattr(L, name).argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    img = np.ascontiguousarray(image, np.float32)
    m = np.ascontiguousarray(model, np.float32)
    return float(L.L2_entropy(width, _p(img), _p(m))), float(L.L2_entropy_gradient(width, _p(img), _p(m)))


# ------------------------------------------------ projected L-BFGS direction

def _lbfgs_fixed(image, g, minvalue):
    """Pixels held fixed: on the positivity bound with the gradient pointing outward."""
    return (np.asarray(image, np.float64) <= minvalue * 1.000001) & (np.asarray(g, np.float64) > 0)


def lbfgs_direction64(S, Y, gamma, image, g, minvalue=1e-8):
    """The batched search's projected L-BFGS direction (method 4), by the C
    oracle's two-loop recursion. S, Y: [count][n] pairs, oldest first; the
    newest LBFGS_PAIRS (4) of them are used, as in the search."""
    L = fp64()
    S = np.ascontiguousarray(S, np.float64)
    Y = np.ascontiguousarray(Y, np.float64)
    img = np.ascontiguousarray(image, np.float64)
    gr = np.ascontiguousarray(g, np.float64)
    count, n = S.shape
    d = np.zeros(n, np.float64)
    L.o64_lbfgs_direction(n, count, _p(S), _p(Y), float(gamma), _p(img), _p(gr), float(minvalue), _p(d))
    return d


def lbfgs_direction_compact(S, Y, gamma, image, g, minvalue=1e-8):
    """The same direction from the compact representation of the inverse BFGS
    matrix (Byrd, Nocedal and Schnabel, 1994):
        H q = gamma q + S^T t + gamma Y^T b,
        b = -R^-1 u,  t = R^-T ((D + gamma Y Y^T) R^-1 u - v),
    u = S q, v = gamma Y q, R = upper triangle of S Y^T, D its diagonal. It
    needs the 2m dots S q, Y q (one pass over q), the m x m products S Y^T and
    Y Y^T (kept as pairs arrive) and one combination pass. All pairs given are
    used (pass the newest LBFGS_PAIRS to match the search): the formulation
    for a device path, where the two-loop recursion would need 2m dependent
    grid-wide reductions."""
    S = np.asarray(S, np.float64)
    Y = np.asarray(Y, np.float64)
    fixed = _lbfgs_fixed(image, g, minvalue)
    q = np.where(fixed, 0.0, np.asarray(g, np.float64))
    if S.shape[0] == 0:
        return np.where(fixed, 0.0, -q)
    SY = S @ Y.T
    R = np.triu(SY)
    D = np.diag(np.diag(SY))
    u = S @ q
    v = gamma * (Y @ q)
    Ru = np.linalg.solve(R, u)
    t = np.linalg.solve(R.T, (D + gamma * (Y @ Y.T)) @ Ru - v)
    Hq = gamma * q + S.T @ t - gamma * (Y.T @ Ru)
    return np.where(fixed, 0.0, -Hq)
