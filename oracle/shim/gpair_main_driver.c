/*
 * gpair_main_driver.c -- entry point around the reference's init_data, plus
 * stand-ins for the symbols gpair.c's main references.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Compiled with the reference's unchanged
 * gpair1/trunk/gpair.c (main renamed by -Dmain=gpair_reference_main), cpu.c
 * and getoifits.c, all read from the reference tree at build time, into
 * oracle/_ref/libgpair_ref_main.so.
 *
 * oracle_ref_init_data fills gpair.c's globals (npow, nbis, oifits_info and
 * the data / data_err / data_phasor arrays; gpair1/trunk/gpair.c:27-52) from
 * plain arrays, calls the reference's init_data (gpair1/trunk/gpair.c:997-1066)
 * and copies the packed arrays out.
 *
 * The gpu_* functions (the OpenCL host layer, gpair1/trunk/gpu.c) and the
 * cfitsio image routines are referenced only from main, writefits and
 * read_fits_image, which the tests never call; their stand-ins report the
 * misuse and abort.
 */
#include <complex.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "getoifits.h"

extern int npow, nbis, nuv, ndof;
extern oi_data oifits_info;
extern float *data, *data_err;
extern float complex *data_phasor;
void init_data(int do_extrapolation);

int oracle_ref_init_data(int do_extrapolation, int n_pow, int n_bis, const float *pow_, const float *powerr,
                         const float *bisamp, const float *bisamperr, const float *bisphs, const float *bisphserr,
                         const int64_t *uvpnt3, float *data_out, float *err_out, float complex *phasor_out)
{
    size_t nd = (size_t)n_pow + 2 * (size_t)n_bis;
    memset(&oifits_info, 0, sizeof(oifits_info));
    oifits_info.pow = malloc(sizeof(float) * (n_pow ? n_pow : 1));
    oifits_info.powerr = malloc(sizeof(float) * (n_pow ? n_pow : 1));
    oifits_info.bisamp = malloc(sizeof(float) * (n_bis ? n_bis : 1));
    oifits_info.bisamperr = malloc(sizeof(float) * (n_bis ? n_bis : 1));
    oifits_info.bisphs = malloc(sizeof(float) * (n_bis ? n_bis : 1));
    oifits_info.bisphserr = malloc(sizeof(float) * (n_bis ? n_bis : 1));
    oifits_info.bsref = calloc(n_bis ? n_bis : 1, sizeof(oi_bsref));
    data = malloc(sizeof(float) * (nd ? nd : 1));
    data_err = malloc(sizeof(float) * (nd ? nd : 1));
    data_phasor = malloc(sizeof(float complex) * (n_bis ? n_bis : 1));
    if (!oifits_info.pow || !oifits_info.powerr || !oifits_info.bisamp || !oifits_info.bisamperr ||
        !oifits_info.bisphs || !oifits_info.bisphserr || !oifits_info.bsref || !data || !data_err || !data_phasor)
        return -1;
    memcpy(oifits_info.pow, pow_, sizeof(float) * n_pow);
    memcpy(oifits_info.powerr, powerr, sizeof(float) * n_pow);
    memcpy(oifits_info.bisamp, bisamp, sizeof(float) * n_bis);
    memcpy(oifits_info.bisamperr, bisamperr, sizeof(float) * n_bis);
    memcpy(oifits_info.bisphs, bisphs, sizeof(float) * n_bis);
    memcpy(oifits_info.bisphserr, bisphserr, sizeof(float) * n_bis);
    for (int t = 0; t < n_bis; t++) {
        oifits_info.bsref[t].ab.uvpnt = (long)uvpnt3[3 * t];
        oifits_info.bsref[t].bc.uvpnt = (long)uvpnt3[3 * t + 1];
        oifits_info.bsref[t].ca.uvpnt = (long)uvpnt3[3 * t + 2];
    }
    oifits_info.npow = n_pow;
    oifits_info.nbis = n_bis;
    npow = n_pow;
    nbis = n_bis;
    ndof = 0;
    fflush(stdout);
    init_data(do_extrapolation);
    fflush(stdout);
    memcpy(data_out, data, sizeof(float) * nd);
    memcpy(err_out, data_err, sizeof(float) * nd);
    memcpy(phasor_out, data_phasor, sizeof(float complex) * n_bis);
    int delta = ndof;
    free(oifits_info.pow); free(oifits_info.powerr); free(oifits_info.bisamp); free(oifits_info.bisamperr);
    free(oifits_info.bisphs); free(oifits_info.bisphserr); free(oifits_info.bsref);
    free(data); free(data_err); free(data_phasor);
    memset(&oifits_info, 0, sizeof(oifits_info));
    data = NULL; data_err = NULL; data_phasor = NULL;
    return delta;
}

static void oracle_unavailable(const char *name)
{
    fprintf(stderr, "oracle: %s is not available in the oracle build of gpair.c\n", name);
    abort();
}

#define STUB(name) void name(void) { oracle_unavailable(#name); }
STUB(gpu_backup_gradient)
STUB(gpu_build_kernels)
STUB(gpu_cleanup)
STUB(gpu_compute_criterion_gradient_curr)
STUB(gpu_compute_criterion_gradient_temp)
STUB(gpu_compute_data_gradient_curr)
STUB(gpu_compute_data_gradient_temp)
STUB(gpu_compute_descent_dir)
STUB(gpu_compute_entropy_gradient_curr)
STUB(gpu_compute_entropy_gradient_temp)
STUB(gpu_copy_data)
STUB(gpu_copy_dft)
STUB(gpu_copy_image)
STUB(gpu_get_chi2_curr)
STUB(gpu_get_chi2_temp)
STUB(gpu_get_entropy_curr)
STUB(gpu_get_entropy_temp)
STUB(gpu_get_image)
STUB(gpu_get_scalprod)
STUB(gpu_getp_ci)
STUB(gpu_getp_dd)
STUB(gpu_getp_fg)
STUB(gpu_getp_fgn)
STUB(gpu_getp_tg)
STUB(gpu_init)
STUB(gpu_linesearch_zoom)
STUB(gpu_shutdown)
STUB(gpu_update_image)
STUB(gpu_update_tempimage)
STUB(fits_create_file)
STUB(fits_create_img)
STUB(fits_read_img)
STUB(fits_read_keys_lng)
STUB(fits_update_key)
STUB(fits_write_img)
