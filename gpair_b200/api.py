"""ctypes bindings of libgpair_b200.so (the C ABI in include/gpair_b200.h).

Everything here calls into the native library; there is no Python or CPU
fallback. If the library is missing, :func:`lib` raises.

* :func:`index_oifits`  -- the OIFITS uv/triangle indexer (get_oi_fits_data,
  gpair1/trunk/getoifits.c:65-357), bit-exact with the reference
* :func:`init_data`, :func:`set_model`, :func:`dft_tables` -- host setup
  (gpair1/trunk/gpair.c:997-1066, gpair1/trunk/cpu.c:645-749,
  gpair1/trunk/gpair.c:231-245)
* :class:`Problem` -- one reconstruction problem as flat arrays
* :class:`Reconstructor` -- a device context: criterion, gradient, device CG
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .oifits import OIFits

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgpair_b200.so")

GPAIR_OK = 0
PREC_FP32, PREC_SPLIT16, PREC_TF32, PREC_TF32X3, PREC_SPLIT16F8 = 0, 1, 2, 3, 4
REG_GULL_SKILLING, REG_L2 = 0, 1
IMG_CURR, IMG_TEMP = 0, 1


class GpairError(RuntimeError):
    pass


class UV(C.Structure):
    _fields_ = [("u", C.c_float), ("v", C.c_float), ("bandwidth", C.c_float), ("wavelength", C.c_float)]


class Float2(C.Structure):
    _fields_ = [("s0", C.c_float), ("s1", C.c_float)]


class Long4(C.Structure):
    _fields_ = [("s0", C.c_int64), ("s1", C.c_int64), ("s2", C.c_int64), ("s3", C.c_int64)]


class Short4(C.Structure):
    _fields_ = [("s0", C.c_int16), ("s1", C.c_int16), ("s2", C.c_int16), ("s3", C.c_int16)]


class OiWavelength(C.Structure):
    _fields_ = [("insname", C.c_char_p), ("nwave", C.c_int), ("eff_wave", C.c_void_p), ("eff_band", C.c_void_p)]


class OiVis2(C.Structure):
    _fields_ = [("insname", C.c_char_p), ("numrec", C.c_long), ("nwave", C.c_int), ("target_id", C.c_void_p),
                ("vis2data", C.c_void_p), ("vis2err", C.c_void_p), ("ucoord", C.c_void_p), ("vcoord", C.c_void_p),
                ("flag", C.c_void_p)]


class OiT3(C.Structure):
    _fields_ = [("insname", C.c_char_p), ("numrec", C.c_long), ("nwave", C.c_int), ("target_id", C.c_void_p),
                ("t3amp", C.c_void_p), ("t3amperr", C.c_void_p), ("t3phi", C.c_void_p), ("t3phierr", C.c_void_p),
                ("u1coord", C.c_void_p), ("v1coord", C.c_void_p), ("u2coord", C.c_void_p), ("v2coord", C.c_void_p),
                ("flag", C.c_void_p)]


class OiData(C.Structure):
    _fields_ = [("npow", C.c_int), ("nbis", C.c_int), ("nuv", C.c_int),
                ("pow", C.POINTER(C.c_float)), ("powerr", C.POINTER(C.c_float)),
                ("bisamp", C.POINTER(C.c_float)), ("bisamperr", C.POINTER(C.c_float)),
                ("bisphs", C.POINTER(C.c_float)), ("bisphserr", C.POINTER(C.c_float)),
                ("uv", C.POINTER(UV)), ("uvpnt", C.POINTER(C.c_int64)), ("sign", C.POINTER(C.c_int16))]


class CgParams(C.Structure):
    _fields_ = [("method", C.c_int), ("iterations", C.c_int), ("alpha", C.c_float), ("minvalue", C.c_double),
                ("wolfe1", C.c_double), ("wolfe2", C.c_double), ("step_max", C.c_double), ("max_zoom", C.c_int),
                ("max_bracket", C.c_int), ("resume", C.c_int), ("host_loop", C.c_int),
                ("line_search", C.c_int), ("target_J", C.c_double), ("batch_step_max", C.c_double),
                ("stop_flag", C.c_void_p)]


LS_WOLFE, LS_BATCH, LS_TRIALS = 0, 1, 8
BATCH_INDEPENDENT = 1  # gpair_batch_create_ex flag: independent branches, no lockstep grouping
BATCH_FORWARDS_ONLY = 2  # gpair_batch_create_ex flag: lockstep with grouped trial forwards only
BATCH_STAGE_STAMPS = 4  # gpair_batch_create_ex flag: device timer stamps between the staged launches


def batch_prep_passes(p: int) -> int:
    """gpair_batch_create_ex flag GPAIR_BATCH_PREP_PASSES(p): passes of image rows per block of a
    staged batch's trial prep (0: chosen by the batch)."""
    return (p & 63) << 8
TUNE_PRECISION, TUNE_SPLITS, TUNE_CACHE, TUNE_BATCHED, TUNE_TILE = 1, 2, 4, 8, 16
TUNE_MAX_CANDIDATES = 16


class TuneResult(C.Structure):
    _fields_ = [("precision", C.c_int), ("adjoint_splits", C.c_int), ("ms_per_eval", C.c_double),
                ("from_cache", C.c_int), ("n_candidates", C.c_int), ("tile_m", C.c_int),
                ("cand_precision", C.c_int * TUNE_MAX_CANDIDATES), ("cand_splits", C.c_int * TUNE_MAX_CANDIDATES),
                ("cand_tile_m", C.c_int * TUNE_MAX_CANDIDATES), ("cand_ms", C.c_double * TUNE_MAX_CANDIDATES)]


class CgResult(C.Structure):
    _fields_ = [("iterations_done", C.c_int), ("criterion_evals", C.c_int), ("grad_evals", C.c_int),
                ("J", C.c_double), ("chi2", C.c_double), ("entropy", C.c_double), ("last_step", C.c_double),
                ("last_beta", C.c_double), ("status", C.c_int), ("reached", C.c_int), ("stopped", C.c_int)]


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GpairError(f"{LIB_PATH} is missing: run `python -m gpair_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
        L.gpair_strerror.restype = C.c_char_p
        L.gpair_last_error.restype = C.c_char_p
        L.gpair_last_error.argtypes = [vp]
        L.gpair_create.argtypes = [C.POINTER(vp), i]
        L.gpair_destroy.argtypes = [vp]
        L.gpair_set_problem.argtypes = [vp, i, f, i, vp, i, i, vp, vp, vp, vp, vp, vp]
        L.gpair_set_precision.argtypes = [vp, i]
        L.gpair_get_precision.argtypes = [vp]
        L.gpair_set_image.argtypes = [vp, i, vp]
        L.gpair_get_image.argtypes = [vp, i, vp]
        L.gpair_criterion.argtypes = [vp, i, C.POINTER(d), C.POINTER(d)]
        L.gpair_gradient.argtypes = [vp, i, f]
        for name in ("gpair_get_visibilities", "gpair_get_mock", "gpair_get_data_gradient",
                     "gpair_get_entropy_gradient"):
            getattr(L, name).argtypes = [vp, vp]
        L.gpair_get_full_gradient.argtypes = [vp, i, vp]
        L.gpair_cg_default_params.argtypes = [C.POINTER(CgParams)]
        L.gpair_cg_run.argtypes = [vp, C.POINTER(CgParams), C.POINTER(CgResult), vp, vp, vp, vp, vp]
        L.gpair_last_run_stats.argtypes = [vp, C.POINTER(d), C.POINTER(d), C.POINTER(i)]
        L.gpair_time_stages.argtypes = [vp, i, C.POINTER(d), i]
        L.gpair_time_batch_stages.argtypes = [vp, i, C.POINTER(d), i]
        L.gpair_set_stage_timing.argtypes = [vp, i]
        L.gpair_set_tc_wait.argtypes = [vp, C.c_longlong, i]
        L.gpair_set_tc_pair.argtypes = [vp, i]
        L.gpair_set_pdl.argtypes = [vp, i]
        L.gpair_set_shared_splits.argtypes = [vp, i]
        L.gpair_get_tc_pair.argtypes = [vp]
        L.gpair_last_run_stage_ms.argtypes = [vp, C.POINTER(d), C.POINTER(i), i]
        L.gpair_get_oi_fits_data.argtypes = [i, f, f, i, vp, i, vp, i, vp, C.POINTER(OiData)]
        L.gpair_free_oi_data.argtypes = [C.POINTER(OiData)]
        L.gpair_init_data.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.gpair_set_model.argtypes = [i, f, i, f, f, vp]
        L.gpair_dft_tables.argtypes = [i, i, vp, f, vp, vp, vp, vp, i]
        L.gpair_set_exit_on_error.argtypes = [i]
        L.gpair_adjoint_image.argtypes = [vp, vp, vp]
        L.gpair_stop_flag_create.argtypes = [C.POINTER(vp)]
        L.gpair_set_regularizer.argtypes = [vp, i]
        L.gpair_cg_checkpoint_size.argtypes = [vp]
        L.gpair_cg_checkpoint_size.restype = C.c_size_t
        L.gpair_cg_checkpoint_save.argtypes = [vp, vp, C.c_size_t]
        L.gpair_cg_checkpoint_load.argtypes = [vp, vp, C.c_size_t]
        L.gpair_autotune.argtypes = [vp, i, i, C.POINTER(TuneResult)]
        L.gpair_update_pixel.argtypes = [vp, i, i, f, C.POINTER(d), C.POINTER(d)]
        L.gpair_batch_create.argtypes = [C.POINTER(vp), C.POINTER(vp), i, i]
        L.gpair_batch_create_ex.argtypes = [C.POINTER(vp), C.POINTER(vp), i, i, i]
        L.gpair_batch_grouped.argtypes = [vp]
        L.gpair_batch_prep_passes.argtypes = [vp]
        L.gpair_batch_stage_stamps.argtypes = [vp, vp, i, i]
        L.gpair_batch_run.argtypes = [vp, C.POINTER(CgParams), C.POINTER(CgResult)]
        L.gpair_batch_destroy.argtypes = [vp]
        L.gpair_cg_run_many.argtypes = [C.POINTER(vp), i, C.POINTER(CgParams), C.POINTER(CgResult)]
        L.gpair_stop_flag_reset.argtypes = [vp]
        L.gpair_stop_flag_destroy.argtypes = [vp]
        L.gpair_global_context.restype = vp
        _declare_reference_boundary(L)
        _lib = L
    return _lib


def _declare_reference_boundary(L):
    """Prototypes of the reference-boundary functions (gpair1/trunk/gpu.h:5-120)."""
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    proto = {
        "print_opencl_error": (None, [C.c_char_p, i]),
        "print_cl_errstring": (C.c_char_p, [i]),
        "gpu_backup_gradient": (None, [i, vp, vp]),
        "gpu_build_kernels": (None, [i, i, i]),
        "gpu_check_data": (None, [vp, i, vp, i, vp, i, vp]),
        "gpu_compare_data": (None, [i, vp, vp]),
        "gpu_compare_complex_data": (None, [i, vp, vp]),
        "gpu_compute_criterion_gradient": (None, [i, f, vp]),
        "gpu_compute_criterion_gradient_curr": (None, [i, f]),
        "gpu_compute_criterion_gradient_temp": (None, [i, f]),
        "gpu_compute_criterion_step": (None, [i, f, f]),
        "gpu_compute_entropy": (None, [i, vp, vp]),
        "gpu_compute_entropy_gradient": (None, [i, vp]),
        "gpu_compute_entropy_gradient_curr": (None, [i]),
        "gpu_compute_entropy_gradient_temp": (None, [i]),
        "gpu_compute_flux": (None, [vp, vp, vp]),
        "gpu_compute_data_gradient": (None, [vp, i, i, i, i]),
        "gpu_compute_data_gradient_curr": (None, [i, i, i, i]),
        "gpu_compute_data_gradient_temp": (None, [i, i, i, i]),
        "gpu_compute_descent_dir": (None, [i, f]),
        "gpu_copy_data": (None, [vp, vp, i, i, vp, i, i, vp, vp, i, vp, i, i]),
        "gpu_copy_dft": (None, [vp, vp, i]),
        "gpu_copy_image": (None, [vp, i, i]),
        "gpu_cleanup": (None, []),
        "gpu_data2chi2": (None, [i]),
        "gpu_error_callback": (i, [C.c_char_p]),
        "gpu_get_chi2_curr": (f, [i, i, i, i, i]),
        "gpu_get_chi2_temp": (f, [i, i, i, i, i]),
        "gpu_get_chi2": (f, [i, i, i, i, i, vp]),
        "gpu_get_entropy": (f, [i, vp]),
        "gpu_get_entropy_curr": (f, [i]),
        "gpu_get_entropy_temp": (f, [i]),
        "gpu_get_image": (vp, [i, vp, vp]),
        "gpu_get_scalprod": (f, [i, i, vp, vp]),
        "gpu_image2chi2": (None, [i, i, i, i, i, vp]),
        "gpu_image2vis": (None, [i, i, vp]),
        "gpu_init": (None, []),
        "gpu_linesearch_zoom": (f, [i, i, i, i, i, i, f, f, f, f, f, vp, vp, vp, vp, f]),
        "gpu_new_chi2": (None, [i, i, i, i]),
        "gpu_vis2data": (None, [vp, i, i, i]),
        "gpu_scalar_prod": (None, [i, i, vp, vp, vp]),
        "gpu_shutdown": (None, []),
        "gpu_update_image": (None, [i, f, f, vp]),
        "gpu_update_tempimage": (None, [i, f, f, vp]),
    }
    for name in ("gpu_getp_ci", "gpu_getp_ti", "gpu_getp_fgn", "gpu_getp_fg", "gpu_getp_dd", "gpu_getp_tg",
                 "gpu_getp_eg"):
        proto[name] = (vp, [])
    proto["gpair_set_zoom_trial_cap"] = (C.c_int, [i])
    proto["gpair_zoom_cap_hits"] = (C.c_int, [])
    proto["gpair_zoom_cap_hits_reset"] = (None, [])
    for name, (res, args) in proto.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args



def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _check(rc: int, ctx=None):
    if rc != GPAIR_OK:
        L = lib()
        detail = L.gpair_last_error(ctx).decode() if ctx else ""
        raise GpairError(f"{L.gpair_strerror(rc).decode()} ({rc}) {detail}")


# --------------------------------------------------------------- indexing

@dataclass
class Indexed:
    """Output of the OIFITS indexer (oi_data, gpair1/trunk/getoifits.h:61-75)."""
    npow: int
    nbis: int
    nuv: int
    pow: np.ndarray
    powerr: np.ndarray
    bisamp: np.ndarray
    bisamperr: np.ndarray
    bisphs: np.ndarray
    bisphserr: np.ndarray
    uv: np.ndarray  # float32 [nuv, 4]: u, v, bandwidth, wavelength
    uvpnt: np.ndarray  # int64 [nbis, 3]
    sign: np.ndarray  # int16 [nbis, 3]


def _oifits_structs(oi: OIFits):
    keep = []

    def arr(x, dt):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a

    waves = (OiWavelength * max(1, len(oi.wavelengths)))()
    for j, w in enumerate(oi.wavelengths):
        name = w.insname.encode()
        keep.append(name)
        waves[j] = OiWavelength(name, len(w.eff_wave), _p(arr(w.eff_wave, np.float32)), _p(arr(w.eff_band, np.float32)))
    vis2 = (OiVis2 * max(1, len(oi.vis2)))()
    for j, t in enumerate(oi.vis2):
        name = t.insname.encode()
        keep.append(name)
        vis2[j] = OiVis2(name, len(t.ucoord), t.nwave, _p(arr(t.target_id, np.int32)), _p(arr(t.vis2data, np.float64)),
                         _p(arr(t.vis2err, np.float64)), _p(arr(t.ucoord, np.float64)), _p(arr(t.vcoord, np.float64)),
                         _p(arr(t.flag, np.uint8)))
    t3s = (OiT3 * max(1, len(oi.t3)))()
    for j, t in enumerate(oi.t3):
        name = t.insname.encode()
        keep.append(name)
        t3s[j] = OiT3(name, len(t.u1coord), t.nwave, _p(arr(t.target_id, np.int32)), _p(arr(t.t3amp, np.float64)),
                      _p(arr(t.t3amperr, np.float64)), _p(arr(t.t3phi, np.float64)), _p(arr(t.t3phierr, np.float64)),
                      _p(arr(t.u1coord, np.float64)), _p(arr(t.v1coord, np.float64)), _p(arr(t.u2coord, np.float64)),
                      _p(arr(t.v2coord, np.float64)), _p(arr(t.flag, np.uint8)))
    return waves, vis2, t3s, keep


def index_oifits(oi: OIFits, minband: float = 0.0, maxband: float = 1e30, target_id: Optional[int] = None) -> Indexed:
    """uv list and triangle references of an OIFITS data set (band limits in nm)."""
    L = lib()
    waves, vis2, t3s, keep = _oifits_structs(oi)
    out = OiData()
    rc = L.gpair_get_oi_fits_data(oi.target_id if target_id is None else target_id, minband, maxband,
                                  len(oi.wavelengths), C.addressof(waves), len(oi.vis2), C.addressof(vis2),
                                  len(oi.t3), C.addressof(t3s), C.byref(out))
    _check(rc)
    try:
        def grab(ptr, n, dt, shape=None):
            if n == 0:
                return np.zeros(shape or (0,), dt)
            a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
            return a.reshape(shape) if shape else a
        npow, nbis, nuv = out.npow, out.nbis, out.nuv
        uv = (np.ctypeslib.as_array(C.cast(out.uv, C.POINTER(C.c_float)), shape=(nuv * 4,)).copy().reshape(nuv, 4)
              if nuv else np.zeros((0, 4), np.float32))
        res = Indexed(npow, nbis, nuv, grab(out.pow, npow, np.float32), grab(out.powerr, npow, np.float32),
                      grab(out.bisamp, nbis, np.float32), grab(out.bisamperr, nbis, np.float32),
                      grab(out.bisphs, nbis, np.float32), grab(out.bisphserr, nbis, np.float32), uv,
                      grab(out.uvpnt, 3 * nbis, np.int64, (nbis, 3)), grab(out.sign, 3 * nbis, np.int16, (nbis, 3)))
    finally:
        L.gpair_free_oi_data(C.byref(out))
    del keep
    return res


def init_data(ix: Indexed, do_extrapolation: int = 1):
    """data, data_err, phasor (complex64), ndof change -- gpair1/trunk/gpair.c:997-1066."""
    L = lib()
    nd = ix.npow + 2 * ix.nbis
    data = np.zeros(max(nd, 1), np.float32)
    err = np.zeros(max(nd, 1), np.float32)
    ph = np.zeros(max(ix.nbis, 1), np.complex64)
    bisamp = ix.bisamp.copy()
    bisamperr = ix.bisamperr.copy()
    uvpnt = np.ascontiguousarray(ix.uvpnt, np.int64)
    delta = L.gpair_init_data(do_extrapolation, ix.npow, ix.nbis, _p(ix.pow), _p(ix.powerr), _p(bisamp),
                              _p(bisamperr), _p(ix.bisphs), _p(ix.bisphserr), _p(uvpnt), _p(data), _p(err), _p(ph))
    return data[:nd], err[:nd], ph[:ix.nbis], int(delta)


def set_model(width: int, pixellation: float, modeltype: int, modelwidth: float, modelflux: float) -> np.ndarray:
    m = np.zeros(width * width, np.float32)
    _check(lib().gpair_set_model(width, pixellation, modeltype, modelwidth, modelflux, _p(m)))
    return m


def dft_tables(width: int, uv: np.ndarray, pixellation: float, transposed: bool = False):
    """Reference DFT tables: CPU layout [nuv][N] complex64 (and the padded [N][nuv] GPU layout)."""
    uv = np.ascontiguousarray(uv, np.float32)
    nuv = uv.shape[0]
    tx = np.zeros(nuv * width, np.complex64)
    ty = np.zeros(nuv * width, np.complex64)
    if transposed:
        alloc = 1 << int(np.ceil(np.log2(max(nuv * width, 1))))
        gx = np.zeros(alloc, np.complex64)
        gy = np.zeros(alloc, np.complex64)
        _check(lib().gpair_dft_tables(width, nuv, _p(uv), pixellation, _p(tx), _p(ty), _p(gx), _p(gy), alloc))
        return tx, ty, gx, gy
    _check(lib().gpair_dft_tables(width, nuv, _p(uv), pixellation, _p(tx), _p(ty), None, None, 0))
    return tx, ty


# ---------------------------------------------------------------- problems

@dataclass
class Problem:
    """A reconstruction problem in the reference's flat layout."""
    width: int
    pixellation: float
    uv: np.ndarray  # float32 [nuv, 4]
    npow: int
    nbis: int
    data: np.ndarray  # float32 [npow + 2 nbis]
    data_err: np.ndarray
    phasor: np.ndarray  # complex64 [nbis]
    uvpnt: np.ndarray  # int64 [nbis, 3]
    sign: np.ndarray  # int16 [nbis, 3]
    model: np.ndarray  # float32 [N*N]
    alpha: float = 1e-3

    @property
    def nuv(self) -> int:
        return int(self.uv.shape[0])

    @property
    def npix(self) -> int:
        return self.width * self.width

    def start_image(self) -> np.ndarray:
        """max(prior, 1e-8), gpair1/trunk/gpair.c:217-225."""
        return np.maximum(self.model, np.float32(1e-8)).astype(np.float32)

    def dft_flops(self) -> float:
        """Algorithmic FLOPs of one forward DFT (= one adjoint): 4 N^2 nuv + 8 N nuv."""
        return 4.0 * self.npix * self.nuv + 8.0 * self.width * self.nuv


def problem_from_oifits(oi: OIFits, width: int, pixellation: float, alpha: float = 1e-3, modeltype: int = 0,
                        modelwidth: float = 0.0, modelflux: float = 1.0, minband: float = 0.0,
                        maxband: float = 1e30) -> Problem:
    ix = index_oifits(oi, minband, maxband)
    data, err, ph, _ = init_data(ix, 1)
    model = set_model(width, pixellation, modeltype, modelwidth, modelflux)
    return Problem(width, pixellation, ix.uv, ix.npow, ix.nbis, data, err, ph, ix.uvpnt, ix.sign, model, alpha)


def workload_problem(name: str, scene_seed: int = 1, noise_seed: int = 2, array_seed: int = 3) -> Problem:
    """Seeded synthetic problem for a named workload (see gpair_b200.synth.workload)."""
    from .synth import make_workload_data
    w, oi = make_workload_data(name, scene_seed, noise_seed, array_seed)
    return problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha, modeltype=0, modelflux=w.prior_flux)


# -------------------------------------------------------------- contexts

class Reconstructor:
    """A device context (gpair_ctx) holding one problem."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = C.c_void_p()
        _check(self._L.gpair_create(C.byref(h), device))
        self.h = h
        self.device = device
        self.problem: Optional[Problem] = None

    def close(self):
        if self.h:
            self._L.gpair_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        _check(rc, self.h)

    def set_problem(self, p: Problem):
        uv = np.ascontiguousarray(p.uv, np.float32)
        self._keep = [uv, np.ascontiguousarray(p.data, np.float32), np.ascontiguousarray(p.data_err, np.float32),
                      np.ascontiguousarray(p.phasor, np.complex64), np.ascontiguousarray(p.uvpnt, np.int64),
                      np.ascontiguousarray(p.sign, np.int16), np.ascontiguousarray(p.model, np.float32)]
        k = self._keep
        self._c(self._L.gpair_set_problem(self.h, p.width, p.pixellation, p.nuv, _p(k[0]), p.npow, p.nbis, _p(k[1]),
                                          _p(k[2]), _p(k[3]), _p(k[4]), _p(k[5]), _p(k[6])))
        self.problem = p

    def set_tc_pair(self, on: bool = True):
        """Tensor-core contractions on CTA pairs (cta_group::2) or single CTAs."""
        self._c(self._L.gpair_set_tc_pair(self.h, 1 if on else 0))

    def set_pdl(self, on: bool = True):
        """Programmatic dependent launches of the evaluation chain (default on)."""
        self._c(self._L.gpair_set_pdl(self.h, 1 if on else 0))

    def set_precision(self, mode: int):
        self._c(self._L.gpair_set_precision(self.h, mode))

    def set_image(self, img: np.ndarray, which: int = IMG_CURR):
        a = np.ascontiguousarray(img, np.float32).ravel()
        self._c(self._L.gpair_set_image(self.h, which, _p(a)))

    def get_image(self, which: int = IMG_CURR) -> np.ndarray:
        a = np.empty(self.problem.npix, np.float32)
        self._c(self._L.gpair_get_image(self.h, which, _p(a)))
        return a

    def criterion(self, which: int = IMG_CURR):
        chi2, S = C.c_double(), C.c_double()
        self._c(self._L.gpair_criterion(self.h, which, C.byref(chi2), C.byref(S)))
        return chi2.value, S.value

    def gradient(self, which: int = IMG_CURR, alpha: Optional[float] = None):
        a = self.problem.alpha if alpha is None else alpha
        self._c(self._L.gpair_gradient(self.h, which, a))

    def autotune(self, flags: int = 7, reps: int = 3) -> dict:
        """Time criterion + gradient under candidate configurations (precision path,
        adjoint split-K length, tensor-core tile) and keep the fastest (gpair_autotune)."""
        r = TuneResult()
        self._c(self._L.gpair_autotune(self.h, flags, reps, C.byref(r)))
        return {"precision": r.precision, "adjoint_splits": r.adjoint_splits, "ms_per_eval": r.ms_per_eval,
                "from_cache": bool(r.from_cache), "tile_m": r.tile_m,
                "candidates": [(r.cand_precision[i], r.cand_splits[i], r.cand_tile_m[i], r.cand_ms[i])
                               for i in range(r.n_candidates)]}

    def checkpoint(self) -> bytes:
        """The CG state of this context (gpair_cg_checkpoint_save) as bytes."""
        n = self._L.gpair_cg_checkpoint_size(self.h)
        buf = C.create_string_buffer(n)
        self._c(self._L.gpair_cg_checkpoint_save(self.h, buf, n))
        return buf.raw

    def restore(self, data: bytes):
        """Load a checkpoint of the same problem; continue with cg(..., resume=True)."""
        buf = C.create_string_buffer(data, len(data))
        self._c(self._L.gpair_cg_checkpoint_load(self.h, buf, len(data)))

    def save_checkpoint(self, path: str, meta: Optional[dict] = None):
        """Raw checkpoint at `path` plus a JSON header at `path`.json (sizes, iteration, J)."""
        import json
        data = self.checkpoint()
        with open(path, "wb") as f:
            f.write(data)
        p = self.problem
        head = {"format": "gpair_b200 CG checkpoint v1", "bytes": len(data), "width": p.width, "nuv": p.nuv,
                "npow": p.npow, "nbis": p.nbis}
        head.update(meta or {})
        with open(path + ".json", "w") as f:
            json.dump(head, f, indent=1)

    def load_checkpoint(self, path: str):
        with open(path, "rb") as f:
            self.restore(f.read())

    def set_regularizer(self, kind: int):
        """REG_GULL_SKILLING (default) or REG_L2."""
        self._c(self._L.gpair_set_regularizer(self.h, kind))

    def update_pixel(self, x: int, y: int, value: float):
        """Set pixel (x, y) of the current image; returns the updated (chi2, S)."""
        chi2, S = C.c_double(), C.c_double()
        self._c(self._L.gpair_update_pixel(self.h, x, y, value, C.byref(chi2), C.byref(S)))
        return chi2.value, S.value

    def adjoint_image(self, weights: np.ndarray) -> np.ndarray:
        """Re sum_k w_k Fx[k][x] Fy[k][y] for complex uv weights w (length nuv)."""
        w = np.ascontiguousarray(weights, np.complex64)
        out = np.empty(self.problem.npix, np.float32)
        self._c(self._L.gpair_adjoint_image(self.h, _p(w), _p(out)))
        return out

    def visibilities(self) -> np.ndarray:
        v = np.empty(self.problem.nuv, np.complex64)
        self._c(self._L.gpair_get_visibilities(self.h, _p(v)))
        return v

    def mock(self) -> np.ndarray:
        m = np.empty(self.problem.npow + 2 * self.problem.nbis, np.float32)
        self._c(self._L.gpair_get_mock(self.h, _p(m)))
        return m

    def data_gradient(self) -> np.ndarray:
        g = np.empty(self.problem.npix, np.float32)
        self._c(self._L.gpair_get_data_gradient(self.h, _p(g)))
        return g

    def entropy_gradient(self) -> np.ndarray:
        g = np.empty(self.problem.npix, np.float32)
        self._c(self._L.gpair_get_entropy_gradient(self.h, _p(g)))
        return g

    def full_gradient(self, which: int = IMG_CURR) -> np.ndarray:
        g = np.empty(self.problem.npix, np.float32)
        self._c(self._L.gpair_get_full_gradient(self.h, which, _p(g)))
        return g

    def cg(self, iterations: int, method: int = 2, alpha: Optional[float] = None, trace: bool = False,
           resume: bool = False, **kw):
        prm = CgParams()
        self._L.gpair_cg_default_params(C.byref(prm))
        prm.method = method
        prm.iterations = iterations
        prm.resume = 1 if resume else 0
        prm.alpha = self.problem.alpha if alpha is None else alpha
        if method == 4:
            prm.wolfe2 = 0.9  # quasi-Newton curvature constant (the reference's 0.1 is for CG)
        for k, v in kw.items():
            setattr(prm, k, v)
        res = CgResult()
        tr = [np.zeros(iterations, np.float64) for _ in range(5)] if trace else None
        ptrs = [_p(t) for t in tr] if trace else [None] * 5
        self._c(self._L.gpair_cg_run(self.h, C.byref(prm), C.byref(res), *ptrs))
        out = {"iterations": res.iterations_done, "criterion_evals": res.criterion_evals,
               "grad_evals": res.grad_evals, "J": res.J, "chi2": res.chi2, "entropy": res.entropy,
               "last_step": res.last_step, "last_beta": res.last_beta, "reached": bool(res.reached),
               "stopped": bool(res.stopped)}
        if trace:
            out.update(zip(("trace_J", "trace_chi2", "trace_entropy", "trace_step", "trace_beta"), tr))
        return out

    STAGES = ("prep", "forward_dft", "vis_data", "adj_weights", "adjoint_dft", "grad_finalize")

    def time_stages(self, reps: int = 10) -> dict:
        ms = (C.c_double * 6)()
        n = self._L.gpair_time_stages(self.h, reps, ms, 6)
        if n < 0:
            self._c(n)
        return {k: ms[j] for j, k in enumerate(self.STAGES[:n])}

    BATCH_STAGES = ("trials_prep", "forward_dft_batch", "vis_chi2_batch")

    def time_batch_stages(self, reps: int = 10) -> dict:
        ms = (C.c_double * 3)()
        n = self._L.gpair_time_batch_stages(self.h, reps, ms, 3)
        if n < 0:
            self._c(n)
        return {k: ms[j] for j, k in enumerate(self.BATCH_STAGES[:n])}

    def set_stage_timing(self, on: bool = True):
        self._c(self._L.gpair_set_stage_timing(self.h, 1 if on else 0))

    def last_run_stage_ms(self) -> dict:
        ms = (C.c_double * 6)()
        cnt = (C.c_int * 6)()
        n = self._L.gpair_last_run_stage_ms(self.h, ms, cnt, 6)
        return {k: (ms[j], cnt[j]) for j, k in enumerate(self.STAGES[:n])}

    def last_run_stats(self):
        ms, fl, n = C.c_double(), C.c_double(), C.c_int()
        self._c(self._L.gpair_last_run_stats(self.h, C.byref(ms), C.byref(fl), C.byref(n)))
        return ms.value, fl.value, n.value


class StopFlag:
    """Device flag shared by CG runs racing to a target objective."""

    def __init__(self):
        self._L = lib()
        h = C.c_void_p()
        _check(self._L.gpair_stop_flag_create(C.byref(h)))
        self.ptr = h.value

    def reset(self):
        _check(self._L.gpair_stop_flag_reset(self.ptr))

    def close(self):
        if self.ptr:
            self._L.gpair_stop_flag_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _result_dict(res: CgResult) -> dict:
    return {"iterations": res.iterations_done, "criterion_evals": res.criterion_evals, "grad_evals": res.grad_evals,
            "J": res.J, "chi2": res.chi2, "entropy": res.entropy, "last_step": res.last_step,
            "last_beta": res.last_beta, "reached": bool(res.reached), "stopped": bool(res.stopped),
            "status": res.status}


def cg_many(recs, iterations: int, method: int = 2, alpha: Optional[float] = None, resume: bool = False, **kw):
    """The same CG run on several contexts at once (gpair_cg_run_many): each
    context's graph runs on its own stream. Returns one result dict per context."""
    L = lib()
    n = len(recs)
    prm = CgParams()
    L.gpair_cg_default_params(C.byref(prm))
    prm.method = method
    prm.iterations = iterations
    prm.resume = 1 if resume else 0
    prm.alpha = recs[0].problem.alpha if alpha is None else alpha
    for k, v in kw.items():
        setattr(prm, k, v)
    handles = (C.c_void_p * n)(*[r.h.value for r in recs])
    res = (CgResult * n)()
    _check(L.gpair_cg_run_many(handles, n, C.byref(prm), res))
    return [_result_dict(res[i]) for i in range(n)]


def shared_splits(recs) -> None:
    """gpair_set_shared_splits: adjoint split-K lengths for contexts that run
    together, so that their units jointly fill the GPU instead of each alone."""
    L = lib()
    n = len(recs)
    handles = (C.c_void_p * n)(*[r.h.value for r in recs])
    _check(L.gpair_set_shared_splits(handles, n), recs[0].h)


def tune_batch_layout(recs, problems, candidates=None, iterations: int = 2) -> dict:
    """Chooses one precision path and tile layout for reconstructions that run as
    one staged batch: for each candidate (precision, CTA pairs) every context takes
    it, its adjoint split-K length is autotuned (GPAIR_TUNE_SPLITS, batched
    objective) and set for sharing the GPU (shared_splits), and a staged batch runs
    `iterations` CG iterations from the problems' start images (device time).
    The fastest candidate is applied to the contexts and returned with every
    candidate's time. One candidate for all keeps one grouped launch per
    contraction; choosing per instance splits the launches by class."""
    if candidates is None:
        candidates = [(PREC_SPLIT16F8, False), (PREC_SPLIT16F8, True), (PREC_SPLIT16, False), (PREC_SPLIT16, True)]
    times = {}

    def take(prec, pair):
        for r, p in zip(recs, problems):
            r.set_tc_pair(pair)
            r.set_precision(prec)
            r.set_image(p.start_image())
        for r in recs:
            r.autotune(TUNE_SPLITS | TUNE_CACHE | TUNE_BATCHED, reps=2)
        shared_splits(recs)

    for prec, pair in candidates:
        take(prec, pair)
        with Batch(recs, line_search=LS_BATCH) as b:
            for r, p in zip(recs, problems):
                r.set_image(p.start_image())
            b.run(1)  # first launch
            for r, p in zip(recs, problems):
                r.set_image(p.start_image())
            b.run(iterations)
            times[(prec, pair)] = recs[0].last_run_stats()[0]
    best = min(times, key=times.get)
    take(*best)
    for r, p in zip(recs, problems):
        r.set_image(p.start_image())
    return {"precision": best[0], "tc_pair": best[1],
            "candidates_ms": [{"precision": k[0], "tc_pair": k[1], "ms": v} for k, v in times.items()],
            "iterations": iterations}


class Batch:
    """Many reconstructions in one CUDA graph launch (gpair_batch_*). With the
    batched line search and the contexts on tensor-core paths the instances run in
    lockstep: `grouped` is 2 when every stage of an iteration is one launch over all
    instances and every contraction one grouped tcgen05 launch per class (staged),
    1 when only the trial forwards are grouped (forwards_only=True, or instances
    that cannot all be staged), 0 when every context's whole CG loop is an
    independent branch of the graph (independent=True, or no tensor-core context).
    Build after the contexts hold their problems, images and configuration."""

    def __init__(self, recs, line_search: int = LS_BATCH, independent: bool = False, forwards_only: bool = False,
                 stamps: bool = False, prep_passes: int = 0):
        self._L = lib()
        self.recs = list(recs)
        self.line_search = line_search
        h = C.c_void_p()
        arr = (C.c_void_p * len(self.recs))(*[r.h.value for r in self.recs])
        flags = ((BATCH_INDEPENDENT if independent else 0) | (BATCH_FORWARDS_ONLY if forwards_only else 0) |
                 (BATCH_STAGE_STAMPS if stamps else 0) | batch_prep_passes(prep_passes))
        _check(self._L.gpair_batch_create_ex(C.byref(h), arr, len(self.recs), line_search, flags), self.recs[0].h)
        self.h = h
        self.grouped = int(self._L.gpair_batch_grouped(self.h))
        self.prep_passes = int(self._L.gpair_batch_prep_passes(self.h))  # 0: not staged

    def run(self, iterations: int, method: int = 2, alpha: Optional[float] = None, resume: bool = False, **kw):
        prm = CgParams()
        self._L.gpair_cg_default_params(C.byref(prm))
        prm.method = method
        prm.iterations = iterations
        prm.resume = 1 if resume else 0
        prm.alpha = self.recs[0].problem.alpha if alpha is None else alpha
        prm.line_search = self.line_search
        for k, v in kw.items():
            setattr(prm, k, v)
        res = (CgResult * len(self.recs))()
        _check(self._L.gpair_batch_run(self.h, C.byref(prm), res), self.recs[0].h)
        return [_result_dict(res[i]) for i in range(len(self.recs))]

    STAMP_NAMES = ["prep", "forward", "vis_data", "adj_weights", "build_w", "adjoint", "grad_finalize",
                   "descent", "route_ls0", "(ls start)", "trials_prep", "trials_forward", "trials_chi2",
                   "route_lsn", "(post start)", "update", "ctrl_end", "route_end"]

    def stage_times_us(self, reset: bool = True) -> dict:
        """Per-launch device time (us) of a staged batch built with stamps=True,
        summed over every iteration and batched evaluation since the last reset
        (each includes one timer kernel's launch); "batched_evaluations" counts
        the batched-evaluation rounds. {} without stamps."""
        buf = np.zeros(39, np.uint64)
        n = self._L.gpair_batch_stage_stamps(self.h, _p(buf), 39, 1 if reset else 0)
        if n <= 0:
            return {}
        out = {}
        for k, name in enumerate(self.STAMP_NAMES):
            if not name.startswith("("):
                out[name] = float(buf[19 + k + 1]) / 1e3
        out["batched_evaluations"] = int(buf[38])
        return out

    def close(self):
        if getattr(self, "h", None):
            self._L.gpair_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
