"""The C ABI library: loads, exports every function include/gpair_b200.h declares,
and behaves without a GPU (no compute calls here)."""
import ctypes as C
import os
import re
import subprocess

import pytest

import gpair_b200 as g

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gpair_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n.startswith(("gpu_", "gpair_", "print_"))))


def test_header_declares_reference_boundary():
    names = declared_functions()
    # every function of the reference's gpu.h that is not OpenCL-specific
    for n in ["gpu_backup_gradient", "gpu_build_kernels", "gpu_check_data", "gpu_compare_data",
              "gpu_compare_complex_data", "gpu_compute_criterion_gradient", "gpu_compute_criterion_gradient_curr",
              "gpu_compute_criterion_gradient_temp", "gpu_compute_criterion_step", "gpu_compute_entropy",
              "gpu_compute_entropy_gradient", "gpu_compute_entropy_gradient_curr",
              "gpu_compute_entropy_gradient_temp", "gpu_compute_flux", "gpu_compute_data_gradient",
              "gpu_compute_data_gradient_curr", "gpu_compute_data_gradient_temp", "gpu_compute_descent_dir",
              "gpu_copy_data", "gpu_copy_dft", "gpu_copy_image", "gpu_cleanup", "gpu_data2chi2",
              "gpu_error_callback", "gpu_get_chi2_curr", "gpu_get_chi2_temp", "gpu_get_chi2", "gpu_get_entropy",
              "gpu_get_entropy_curr", "gpu_get_entropy_temp", "gpu_get_image", "gpu_get_scalprod", "gpu_getp_ci",
              "gpu_getp_ti", "gpu_getp_fgn", "gpu_getp_fg", "gpu_getp_dd", "gpu_getp_tg", "gpu_getp_eg",
              "gpu_image2chi2", "gpu_image2vis", "gpu_init", "gpu_linesearch_zoom", "gpu_new_chi2",
              "gpu_vis2data", "gpu_scalar_prod", "gpu_shutdown", "gpu_update_image", "gpu_update_tempimage",
              "print_opencl_error", "print_cl_errstring"]:
        assert n in names, n


def test_library_exports_every_declared_function():
    lib = g.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", lib._name], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)


def test_status_strings():
    lib = g.lib()
    assert lib.gpair_strerror(0) == b"GPAIR_OK"
    assert lib.gpair_strerror(-1) == b"GPAIR_ERR_INVALID"
    assert lib.gpair_strerror(-99) == b"GPAIR_ERR_UNKNOWN"


def test_create_without_gpu_reports_no_device():
    from conftest import cuda_device_ok
    if cuda_device_ok():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = g.lib().gpair_create(C.byref(h), 0)
    assert rc == -6  # GPAIR_ERR_NO_DEVICE
    assert not h.value


def test_library_is_built_for_sm100a_only():
    # the build passes -gencode arch=compute_100a,code=sm_100a and nothing else
    from gpair_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_batch_flags_are_checked_before_any_context_is_touched():
    """gpair_batch_create_ex refuses unknown flag bits and a trial-prep pass count
    that is not a power of two (GPAIR_ERR_INVALID) before it reads a context; a
    valid pass count then reaches the context check (a null context:
    GPAIR_ERR_STATE). No GPU call is made."""
    from gpair_b200 import api
    lib = g.lib()
    b = C.c_void_p()
    arr = (C.c_void_p * 1)(None)
    assert api.batch_prep_passes(4) == 4 << 8
    for flags in (api.batch_prep_passes(3), api.batch_prep_passes(6), 1 << 14, 1 << 3):
        assert lib.gpair_batch_create_ex(C.byref(b), arr, 1, api.LS_BATCH, flags) == -1, flags  # INVALID
        assert not b.value
    for p in (0, 1, 2, 4, 8, 16, 32):
        assert lib.gpair_batch_create_ex(C.byref(b), arr, 1, api.LS_BATCH, api.batch_prep_passes(p)) == -4, p
        assert not b.value
    assert lib.gpair_batch_prep_passes(None) == 0
