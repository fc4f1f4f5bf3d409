/*
 * oi_setup.c -- host-side problem setup of the reconstruction path.
 *
 *   gpair_init_data   init_data, gpair1/trunk/gpair.c:997-1066
 *   gpair_set_model   set_model, gpair1/trunk/cpu.c:645-749
 *   gpair_dft_tables  DFT table build, gpair1/trunk/gpair.c:231-245, and the
 *                     transposed device layout of gpair1/trunk/gpair.c:610-636
 *
 * These run once per problem. They keep the reference's float/double mix so
 * that their outputs are bit-identical to the reference's (checked in tests
 * against the oracle's replicas and the reference's own cpu.c).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "gpair_b200.h"

#define SETUP_PI 3.14159265358979323

static float sq(float x) { return x * x; }

int gpair_init_data(int do_extrapolation, int npow, int nbis, const float *pow, const float *powerr,
                    float *bisamp, float *bisamperr, const float *bisphs, const float *bisphserr,
                    const int64_t *uvpnt, float *data, float *data_err, gpair_float2 *phasor)
{
    int ndof_delta = 0;
    for (int ii = 0; ii < npow; ii++) {
        data[ii] = pow[ii];
        data_err[ii] = 1. / fabs(powerr[ii]);
    }
    for (int ii = 0; ii < nbis; ii++) {
        /* missing triple amplitudes: derive them from the three V2 points */
        if ((do_extrapolation == 1) && ((bisamperr[ii] <= 0.) || (bisamperr[ii] > 1e3))) {
            int64_t ab = uvpnt[3 * ii], bc = uvpnt[3 * ii + 1], ca = uvpnt[3 * ii + 2];
            if ((ab < npow) && (bc < npow) && (ca < npow)) {
                float p1 = pow[ab], e1 = powerr[ab], p2 = pow[bc], e2 = powerr[bc], p3 = pow[ca], e3 = powerr[ca];
                float a1 = (p1 + sqrt(sq(p1) + 2.0 * sq(e1))) / 2.;
                float s1 = 1. / (1. / a1 + 2. * (3. * a1 - p1) / sq(e1));
                float a2 = (p2 + sqrt(sq(p2) + 2.0 * sq(e2))) / 2.;
                float s2 = 1. / (1. / a2 + 2. * (3. * a2 - p2) / sq(e2));
                float a3 = (p3 + sqrt(sq(p3) + 2.0 * sq(e3))) / 2.;
                float s3 = 1. / (1. / a3 + 2. * (3. * a3 - p3) / sq(e3));
                bisamp[ii] = sqrt(a1 * a2 * a3);
                bisamperr[ii] = bisamp[ii] * sqrt(s1 / a1 + s2 / a2 + s3 / a3);
            } else {
                bisamp[ii] = 1.0;
                bisamperr[ii] = 1e99;
                ndof_delta--;
            }
        }
        data[npow + 2 * ii] = fabs(bisamp[ii]);
        data[npow + 2 * ii + 1] = 0.;
        data_err[npow + 2 * ii] = 1. / bisamperr[ii];
        data_err[npow + 2 * ii + 1] = 1. / fabs(bisamp[ii] * bisphserr[ii] * SETUP_PI / 180.);
        float complex ph = cexp(-I * bisphs[ii] * SETUP_PI / 180.);
        phasor[ii].s0 = crealf(ph);
        phasor[ii].s1 = cimagf(ph);
    }
    return ndof_delta;
}

int gpair_set_model(int image_width, float image_pixellation, int modeltype, float modelwidth, float modelflux,
                    float *default_model)
{
    if (image_width <= 0 || !default_model) return GPAIR_ERR_INVALID;
    const int N = image_width;
    float flux = 0.0;
    switch (modeltype) {
    case 0: { /* flat */
        float norm = ((float)N * (float)N);
        for (int i = 0; i < N * N; i++) default_model[i] = modelflux / norm;
        break;
    }
    case 1: /* centred Dirac on a 1e-8 floor */
        for (int i = 0; i < N * N; i++) default_model[i] = 1e-8;
        default_model[(N * (N + 1)) / 2] = modelflux;
        break;
    case 2: { /* centred uniform disk, radius modelwidth (mas) */
        float rsq;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) {
                rsq = sq((float)(N / 2 - i)) + sq((float)(N / 2 - j));
                default_model[j * N + i] = (sqrt(rsq) <= (modelwidth / image_pixellation)) ? 1. : 1e-8;
                flux += default_model[j * N + i];
            }
        for (int i = 0; i < N * N; i++) default_model[i] *= modelflux / flux;
        break;
    }
    case 3: { /* Gaussian of FWHM modelwidth; the reference centres it 80 px below the middle */
        float sigma = modelwidth / (2. * sqrt(2. * log(2.)));
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) {
                default_model[j * N + i] = exp(-(sq((float)N / 2 - i) + sq((float)N / 2 - j - 80))
                                               / (2. * sq(sigma / image_pixellation)));
                flux += default_model[j * N + i];
            }
        for (int i = 0; i < N * N; i++) default_model[i] *= modelflux / flux;
        break;
    }
    case 4: { /* Lorentzian */
        float sigma = modelwidth;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) {
                default_model[j * N + i] = sigma / (sq(sigma) + sq((float)N / 2 - i) + sq((float)N / 2 - j));
                flux += default_model[j * N + i];
            }
        for (int i = 0; i < N * N; i++) default_model[i] *= modelflux / flux;
        break;
    }
    default:
        return GPAIR_ERR_INVALID; /* the reference leaves the buffer untouched */
    }
    return GPAIR_OK;
}

int gpair_dft_tables(int image_width, int nuv, const gpair_uv *uv, float pixellation, gpair_float2 *dft_x,
                     gpair_float2 *dft_y, gpair_float2 *dft_x_t, gpair_float2 *dft_y_t, int dft_alloc)
{
    const int N = image_width;
    if (N <= 0 || nuv < 0 || !uv || !dft_x || !dft_y) return GPAIR_ERR_INVALID;
    if ((dft_x_t || dft_y_t) && (int64_t)dft_alloc < (int64_t)nuv * N) return GPAIR_ERR_INVALID;
    for (int uu = 0; uu < nuv; uu++) {
        for (int ii = 0; ii < N; ii++) {
            /* phase in double, same factor order as the reference's expression */
            float complex ex = cexp(2.0 * I * SETUP_PI * (3.14159265358979323 / 180.0) / 3600000.0 * pixellation
                                    * uv[uu].u * (float)ii);
            float complex ey = cexp(-2.0 * I * SETUP_PI * (3.14159265358979323 / 180.0) / 3600000.0 * pixellation
                                    * uv[uu].v * (float)ii);
            dft_x[N * uu + ii].s0 = crealf(ex);
            dft_x[N * uu + ii].s1 = cimagf(ex);
            dft_y[N * uu + ii].s0 = crealf(ey);
            dft_y[N * uu + ii].s1 = cimagf(ey);
        }
    }
    if (dft_x_t && dft_y_t) {
        for (int i = 0; i < dft_alloc; i++) {
            dft_x_t[i].s0 = dft_x_t[i].s1 = 0;
            dft_y_t[i].s0 = dft_y_t[i].s1 = 0;
        }
        for (int uu = 0; uu < nuv; uu++)
            for (int ii = 0; ii < N; ii++) {
                dft_x_t[nuv * ii + uu] = dft_x[N * uu + ii];
                dft_y_t[nuv * ii + uu] = dft_y[N * uu + ii];
            }
    }
    return GPAIR_OK;
}
