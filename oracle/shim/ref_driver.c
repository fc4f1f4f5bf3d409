/*
 * ref_driver.c -- flat C entry points around the reference's own CPU code.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Compiled together with the reference's
 * unchanged gpair1/trunk/cpu.c and gpair1/trunk/getoifits.c (read from the
 * reference tree at build time, never copied) into oracle/_ref/libgpair_ref.so.
 * The wrappers only marshal plain arrays into the reference's structs
 * (chi2_info, oi_data; gpair1/trunk/data_types.h:10-32,
 * gpair1/trunk/getoifits.h:37-75) and call:
 *   get_oi_fits_data        gpair1/trunk/getoifits.c:65-357
 *   image2chi2              gpair1/trunk/cpu.c:435-447
 *   compute_data_gradient   gpair1/trunk/cpu.c:279-369
 *   GullSkilling_entropy(_gradient)  gpair1/trunk/cpu.c:385-412
 *   set_model               gpair1/trunk/cpu.c:645-749
 * image2vis prints a line on every call (gpair1/trunk/cpu.c:460); stdout is
 * sent to /dev/null around the reference calls when `quiet` is set.
 */
#include <fcntl.h>
#include <unistd.h>
#include <stdint.h>
#include "cpu.h"

static oi_data g_data;
static int g_have_data = 0;

static int g_saved_fd = -1;
static void quiet_on(int quiet)
{
    if (!quiet) return;
    fflush(stdout);
    g_saved_fd = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
}
static void quiet_off(int quiet)
{
    if (!quiet || g_saved_fd < 0) return;
    fflush(stdout);
    dup2(g_saved_fd, 1);
    close(g_saved_fd);
    g_saved_fd = -1;
}

/* Run the reference matcher over the tables registered with oracle_shim_*.
 * numvis2/numt3 bound the number of V2 / T3 points (as get_oi_fits_selection
 * would have counted them). Returns the cfitsio-style status. */
int oracle_ref_get_oi_fits_data(int target_id, float minband, float maxband, long numvis2, long numt3,
                                int *npow, int *nbis, int *nuv, int quiet)
{
    if (g_have_data) { free_oi_data(&g_data); g_have_data = 0; }
    oi_usersel usersel;
    memset(&usersel, 0, sizeof(usersel));
    usersel.target_id = target_id;
    usersel.minband = minband;
    usersel.maxband = maxband;
    usersel.numvis2 = numvis2;
    usersel.numt3 = numt3;
    memset(&g_data, 0, sizeof(g_data));
    int status = 0;
    quiet_on(quiet);
    get_oi_fits_data(&usersel, &g_data, &status);
    quiet_off(quiet);
    g_have_data = 1;
    *npow = g_data.npow;
    *nbis = g_data.nbis;
    *nuv = g_data.nuv;
    return status;
}

/* Copy the matcher's output out: uv as [nuv][4] (u, v, bandwidth, wavelength),
 * bsref as [nbis][3] uv indices and signs (ab, bc, ca), data columns as float. */
void oracle_ref_copy_oi_data(float *pow, float *powerr, float *bisamp, float *bisamperr, float *bisphs,
                             float *bisphserr, float *uv, int64_t *uvpnt, int16_t *sign)
{
    for (int i = 0; i < g_data.npow; i++) { pow[i] = g_data.pow[i]; powerr[i] = g_data.powerr[i]; }
    for (int i = 0; i < g_data.nbis; i++) {
        bisamp[i] = g_data.bisamp[i]; bisamperr[i] = g_data.bisamperr[i];
        bisphs[i] = g_data.bisphs[i]; bisphserr[i] = g_data.bisphserr[i];
        uvpnt[3 * i + 0] = g_data.bsref[i].ab.uvpnt; sign[3 * i + 0] = g_data.bsref[i].ab.sign;
        uvpnt[3 * i + 1] = g_data.bsref[i].bc.uvpnt; sign[3 * i + 1] = g_data.bsref[i].bc.sign;
        uvpnt[3 * i + 2] = g_data.bsref[i].ca.uvpnt; sign[3 * i + 2] = g_data.bsref[i].ca.sign;
    }
    for (int i = 0; i < g_data.nuv; i++) {
        uv[4 * i + 0] = g_data.uv[i].u; uv[4 * i + 1] = g_data.uv[i].v;
        uv[4 * i + 2] = g_data.uv[i].bandwidth; uv[4 * i + 3] = g_data.uv[i].wavelength;
    }
}

/* Problem description handed to the cpu.c wrappers: everything chi2_info needs. */
typedef struct {
    int image_width, nuv, npow, nbis;
    const float *data, *data_err;
    const float *phasor;        /* complex64 [nbis] */
    const int64_t *uvpnt;       /* [nbis][3] */
    const int16_t *sign;        /* [nbis][3] */
    const float *dft_x, *dft_y; /* complex64 [nuv][image_width] (the CPU layout) */
} oracle_ref_problem;

typedef struct {
    chi2_info info;
    oi_data od;
} ref_ctx;

static void build_ctx(const oracle_ref_problem *p, ref_ctx *c, float complex *visi, float *mock)
{
    memset(c, 0, sizeof(*c));
    c->od.npow = p->npow;
    c->od.nbis = p->nbis;
    c->od.nuv = p->nuv;
    c->od.bsref = malloc(sizeof(oi_bsref) * (p->nbis ? p->nbis : 1));
    for (int i = 0; i < p->nbis; i++) {
        c->od.bsref[i].ab.uvpnt = p->uvpnt[3 * i + 0]; c->od.bsref[i].ab.sign = p->sign[3 * i + 0];
        c->od.bsref[i].bc.uvpnt = p->uvpnt[3 * i + 1]; c->od.bsref[i].bc.sign = p->sign[3 * i + 1];
        c->od.bsref[i].ca.uvpnt = p->uvpnt[3 * i + 2]; c->od.bsref[i].ca.sign = p->sign[3 * i + 2];
    }
    c->info.npow = p->npow;
    c->info.nbis = p->nbis;
    c->info.nuv = p->nuv;
    c->info.data = (float *)p->data;
    c->info.data_err = (float *)p->data_err;
    c->info.data_phasor = (float complex *)p->phasor;
    c->info.oifits_info = &c->od;
    c->info.image_width = p->image_width;
    c->info.dft_x = (float complex *)p->dft_x;
    c->info.dft_y = (float complex *)p->dft_y;
    c->info.visi = visi;
    c->info.mock = mock;
}

static void free_ctx(ref_ctx *c) { free(c->od.bsref); }

/* chi2 of `image` (reference image2chi2). visi (complex64 [nuv]) and mock
 * ([npow+2nbis]) receive the reference's intermediate results. */
float oracle_ref_image2chi2(const oracle_ref_problem *p, float *image, float *visi, float *mock, int quiet)
{
    ref_ctx c;
    build_ctx(p, &c, (float complex *)visi, mock);
    quiet_on(quiet);
    float chi2 = image2chi2(&c.info, image);
    quiet_off(quiet);
    free_ctx(&c);
    return chi2;
}

/* Data gradient (reference compute_data_gradient). Uses visi/mock from the
 * preceding oracle_ref_image2chi2 on the same image, as the reference does. */
void oracle_ref_data_gradient(const oracle_ref_problem *p, float *image, float *visi, float *mock, float *grad)
{
    ref_ctx c;
    build_ctx(p, &c, (float complex *)visi, mock);
    compute_data_gradient(&c.info, image, grad);
    free_ctx(&c);
}

float oracle_ref_entropy(int image_width, float *image, float *model)
{
    return GullSkilling_entropy(image_width, image, model);
}

void oracle_ref_entropy_gradient(int image_width, float *image, float *model, float *grad)
{
    GullSkilling_entropy_gradient(image_width, image, model, grad);
}

void oracle_ref_set_model(int image_width, float pixellation, int modeltype, float modelwidth, float modelflux,
                          float *model, int quiet)
{
    quiet_on(quiet);
    set_model(image_width, pixellation, modeltype, modelwidth, modelflux, model);
    quiet_off(quiet);
}
