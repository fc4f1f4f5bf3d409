"""The allocation-free data stage, gpair_vis2data_chi2_noalloc, against the main path.

This entry point is for callers that cannot allocate device memory: a host
program whose own allocator owns the device heap, or a latency-critical loop
where a cudaMalloc could serialise the device. It takes caller-owned device
buffers and keeps its reduction scratch in a fixed device array inside the
library. The test feeds it the visibilities that the existing entry point
(gpair_criterion) computed and checks mock data and chi2 against that entry
point's, on two calls in a row (the second call reuses the scratch that the
first left behind). This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import gpair_b200 as g
from gpair_b200 import synth

pytestmark = pytest.mark.gpu


def _entry():
    L = g.lib()
    f = L.gpair_vis2data_chi2_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _device_inputs(p, visi):
    import torch

    dev = torch.device("cuda", 0)
    uv4 = np.zeros((p.nbis, 4), np.int64)
    uv4[:, :3] = p.uvpnt
    sg4 = np.zeros((p.nbis, 4), np.int16)
    sg4[:, :3] = p.sign
    return {"visi": torch.from_numpy(visi.view(np.float32).copy()).to(dev),
            "data": torch.from_numpy(p.data.astype(np.float32)).to(dev),
            "err": torch.from_numpy(p.data_err.astype(np.float32)).to(dev),
            "ph": torch.from_numpy(p.phasor.astype(np.complex64).view(np.float32).copy()).to(dev),
            "uv": torch.from_numpy(uv4).to(dev), "sg": torch.from_numpy(sg4).to(dev)}


def _call(f, p, t):
    import torch

    dev = torch.device("cuda", 0)
    nd = p.npow + 2 * p.nbis
    t_mock = torch.full((nd,), float("nan"), dtype=torch.float32, device=dev)
    t_chi2 = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = f(t["visi"].data_ptr(), p.nuv, p.npow, p.nbis, t["data"].data_ptr(), t["err"].data_ptr(),
           t["ph"].data_ptr(), t["uv"].data_ptr(), t["sg"].data_ptr(), t_mock.data_ptr(), t_chi2.data_ptr(),
           stream.cuda_stream)
    stream.synchronize()
    return rc, t_mock.cpu().numpy(), float(t_chi2.cpu().numpy()[0])


def test_noalloc_flags_an_out_of_range_triangle_then_recovers():
    """A triangle that names a uv point >= nuv is not read and makes chi2 NaN; the
    next clean call starts from a cleared error word and returns a finite chi2."""
    w, oi = synth.make_workload_data("tiny", 1, 2, 3)
    p = g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha)
    with g.Reconstructor(0) as rec:
        rec.set_problem(p)
        rec.set_image(p.start_image())
        chi2_ref, _ = rec.criterion()
        visi = rec.visibilities()
    f = _entry()
    t = _device_inputs(p, visi)
    good = t["uv"].clone()
    t["uv"][p.nbis // 2, 1] = p.nuv  # one past the end
    rc, _, chi2 = _call(f, p, t)
    assert rc == 0 and np.isnan(chi2)
    t["uv"] = good
    rc, _, chi2 = _call(f, p, t)
    assert rc == 0 and np.isfinite(chi2) and abs(chi2 - chi2_ref) / chi2_ref <= 1e-5


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_noalloc_matches_existing_entry_point_twice(name):
    import torch

    w, oi = synth.make_workload_data(name, 1, 2, 3)
    p = g.problem_from_oifits(oi, w.image_width, w.pixellation_mas, w.alpha)
    rng = np.random.default_rng(11)
    img = (p.start_image() * (1 + rng.uniform(0, 2, p.npix))).astype(np.float32)
    with g.Reconstructor(0) as rec:
        rec.set_problem(p)
        rec.set_image(img)
        chi2_ref, _ = rec.criterion()
        visi = rec.visibilities()
        mock_ref = rec.mock()

    dev = torch.device("cuda", 0)
    t_visi = torch.from_numpy(visi.view(np.float32).copy()).to(dev)
    t_data = torch.from_numpy(p.data.astype(np.float32)).to(dev)
    t_err = torch.from_numpy(p.data_err.astype(np.float32)).to(dev)
    t_ph = torch.from_numpy(p.phasor.astype(np.complex64).view(np.float32).copy()).to(dev)
    uv4 = np.zeros((p.nbis, 4), np.int64)
    uv4[:, :3] = p.uvpnt
    sg4 = np.zeros((p.nbis, 4), np.int16)
    sg4[:, :3] = p.sign
    t_uv = torch.from_numpy(uv4).to(dev)
    t_sg = torch.from_numpy(sg4).to(dev)
    nd = p.npow + 2 * p.nbis
    f = _entry()
    stream = torch.cuda.current_stream(dev)
    results = []
    for _ in range(2):
        t_mock = torch.full((nd,), float("nan"), dtype=torch.float32, device=dev)
        t_chi2 = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        rc = f(t_visi.data_ptr(), p.nuv, p.npow, p.nbis, t_data.data_ptr(), t_err.data_ptr(), t_ph.data_ptr(),
               t_uv.data_ptr(), t_sg.data_ptr(), t_mock.data_ptr(), t_chi2.data_ptr(), stream.cuda_stream)
        assert rc == 0
        stream.synchronize()
        mock = t_mock.cpu().numpy()
        chi2 = float(t_chi2.cpu().numpy()[0])
        # the existing entry point forms mock data from FP64 visibilities; this one reads the
        # float visibilities it returned, so agreement is to float rounding (tests' 1e-5 tolerance)
        assert abs(chi2 - chi2_ref) / chi2_ref <= 1e-5
        assert np.allclose(mock, mock_ref, rtol=1e-5, atol=1e-6)
        results.append((mock, chi2))
    assert np.array_equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]


def test_noalloc_rejects_sizes_beyond_its_scratch():
    f = _entry()
    rc = f(None, 3_000_000, 2_000_000, 200_000, None, None, None, None, None, None, C.c_void_p(1), None)
    assert rc == -1  # GPAIR_ERR_INVALID, nothing launched
