/*
 * oifits_mem.c -- in-memory OIFITS tables behind the cfitsio entry points that
 * the reference's getoifits.c calls.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Linked with the reference's unchanged
 * gpair1/trunk/getoifits.c so that its uv/triangle matcher
 * (get_oi_fits_data, gpair1/trunk/getoifits.c:65-357) can be run on seeded
 * synthetic tables and on tables parsed from an OIFITS file by the test
 * harness. It replaces the reference's cfitsio-based reader
 * (gpair1/trunk/read_fits.c:228-603): same structs (exchange.h), same
 * ownership (every array handed out is malloc'd, freed by the reference's
 * free_oi_* functions), same end-of-tables signalling (non-zero *status).
 *
 * HDU model: HDU 1 is an empty primary header; HDUs 2.. are the tables in
 * the order they were registered (wavelength, OI_VIS2 and OI_T3 tables).
 */
#include <stdlib.h>
#include <string.h>
#include "fitsio.h"
#include "exchange.h"

enum { MEM_WAVE = 1, MEM_VIS2 = 2, MEM_T3 = 3 };

typedef struct {
    int kind;
    char insname[FLEN_VALUE];
    long numrec;
    int nwave;
    /* wavelength table */
    float *eff_wave, *eff_band;
    /* data tables, row-major [numrec][nwave] for per-channel columns */
    int *target_id;
    double *c0, *c1, *c2, *c3; /* vis2: vis2data, vis2err; t3: t3amp, t3amperr, t3phi, t3phierr */
    double *u1, *v1, *u2, *v2;  /* vis2 uses u1/v1 only */
    char *flag;
} mem_hdu;

#define MEM_MAX_HDU 256
static mem_hdu g_hdu[MEM_MAX_HDU];
static int g_nhdu = 0;      /* number of tables (HDUs 2..g_nhdu+1) */
static int g_cur = 1;       /* current HDU number (1-based) */
static int g_target_id = 1;
static char g_target_name[17] = "SYNTH";
struct oracle_fitsfile { int dummy; };
static struct oracle_fitsfile g_file;

static void *dup_mem(const void *src, size_t n)
{
    void *p = malloc(n ? n : 1);
    if (src && n) memcpy(p, src, n);
    return p;
}

static void free_hdu(mem_hdu *h)
{
    free(h->eff_wave); free(h->eff_band); free(h->target_id);
    free(h->c0); free(h->c1); free(h->c2); free(h->c3);
    free(h->u1); free(h->v1); free(h->u2); free(h->v2); free(h->flag);
    memset(h, 0, sizeof(*h));
}

/* ---- registration API (called through ctypes by the test harness) ---- */

void oracle_shim_reset(int target_id)
{
    for (int i = 0; i < g_nhdu; i++) free_hdu(&g_hdu[i]);
    g_nhdu = 0;
    g_cur = 1;
    g_target_id = target_id;
}

int oracle_shim_add_wavelength(const char *insname, int nwave, const float *eff_wave, const float *eff_band)
{
    if (g_nhdu >= MEM_MAX_HDU) return -1;
    mem_hdu *h = &g_hdu[g_nhdu++];
    memset(h, 0, sizeof(*h));
    h->kind = MEM_WAVE;
    strncpy(h->insname, insname, FLEN_VALUE - 1);
    h->nwave = nwave;
    h->eff_wave = dup_mem(eff_wave, sizeof(float) * nwave);
    h->eff_band = dup_mem(eff_band, sizeof(float) * nwave);
    return g_nhdu + 1;
}

int oracle_shim_add_vis2(const char *insname, long numrec, int nwave, const int *target_id,
                         const double *vis2data, const double *vis2err,
                         const double *ucoord, const double *vcoord, const char *flag)
{
    if (g_nhdu >= MEM_MAX_HDU) return -1;
    mem_hdu *h = &g_hdu[g_nhdu++];
    memset(h, 0, sizeof(*h));
    h->kind = MEM_VIS2;
    strncpy(h->insname, insname, FLEN_VALUE - 1);
    h->numrec = numrec;
    h->nwave = nwave;
    size_t nc = (size_t)numrec * nwave;
    h->target_id = dup_mem(target_id, sizeof(int) * numrec);
    h->c0 = dup_mem(vis2data, sizeof(double) * nc);
    h->c1 = dup_mem(vis2err, sizeof(double) * nc);
    h->u1 = dup_mem(ucoord, sizeof(double) * numrec);
    h->v1 = dup_mem(vcoord, sizeof(double) * numrec);
    h->flag = dup_mem(flag, nc);
    return g_nhdu + 1;
}

int oracle_shim_add_t3(const char *insname, long numrec, int nwave, const int *target_id,
                       const double *t3amp, const double *t3amperr, const double *t3phi, const double *t3phierr,
                       const double *u1coord, const double *v1coord, const double *u2coord, const double *v2coord,
                       const char *flag)
{
    if (g_nhdu >= MEM_MAX_HDU) return -1;
    mem_hdu *h = &g_hdu[g_nhdu++];
    memset(h, 0, sizeof(*h));
    h->kind = MEM_T3;
    strncpy(h->insname, insname, FLEN_VALUE - 1);
    h->numrec = numrec;
    h->nwave = nwave;
    size_t nc = (size_t)numrec * nwave;
    h->target_id = dup_mem(target_id, sizeof(int) * numrec);
    h->c0 = dup_mem(t3amp, sizeof(double) * nc);
    h->c1 = dup_mem(t3amperr, sizeof(double) * nc);
    h->c2 = dup_mem(t3phi, sizeof(double) * nc);
    h->c3 = dup_mem(t3phierr, sizeof(double) * nc);
    h->u1 = dup_mem(u1coord, sizeof(double) * numrec);
    h->v1 = dup_mem(v1coord, sizeof(double) * numrec);
    h->u2 = dup_mem(u2coord, sizeof(double) * numrec);
    h->v2 = dup_mem(v2coord, sizeof(double) * numrec);
    h->flag = dup_mem(flag, nc);
    return g_nhdu + 1;
}

/* ---- cfitsio entry points ---- */

int fits_open_file(fitsfile **fptr, const char *name, int mode, int *status)
{
    (void)name; (void)mode;
    if (*status) return *status;
    *fptr = &g_file;
    g_cur = 1;
    return 0;
}

int fits_close_file(fitsfile *fptr, int *status) { (void)fptr; return *status; }

void fits_report_error(FILE *stream, int status)
{
    if (status && status != END_OF_FILE) fprintf(stream, "oracle fits shim: status %d\n", status);
}

int fits_movabs_hdu(fitsfile *fptr, int hdunum, int *hdutype, int *status)
{
    (void)fptr;
    if (*status) return *status;
    if (hdunum < 1 || hdunum > g_nhdu + 1) return (*status = BAD_HDU_NUM);
    g_cur = hdunum;
    if (hdutype) *hdutype = (hdunum == 1) ? IMAGE_HDU : BINARY_TBL;
    return 0;
}

int fits_movrel_hdu(fitsfile *fptr, int nmove, int *hdutype, int *status)
{
    return fits_movabs_hdu(fptr, g_cur + nmove, hdutype, status);
}

int fits_get_hdu_num(fitsfile *fptr, int *hdunum) { (void)fptr; *hdunum = g_cur; return g_cur; }

int fits_get_num_hdus(fitsfile *fptr, int *nhdu, int *status)
{
    (void)fptr;
    *nhdu = g_nhdu + 1;
    return *status;
}

int fits_read_key(fitsfile *fptr, int datatype, const char *keyname, void *value, char *comment, int *status)
{
    (void)fptr; (void)datatype; (void)comment;
    if (*status) return *status;
    if (strcmp(keyname, "EXTNAME") == 0 && g_cur >= 2) {
        const mem_hdu *h = &g_hdu[g_cur - 2];
        strcpy((char *)value, h->kind == MEM_WAVE ? "OI_WAVELENGTH" : h->kind == MEM_VIS2 ? "OI_VIS2" : "OI_T3");
        return 0;
    }
    return (*status = KEY_NO_EXIST);
}

/* ---- exchange.h readers (replacing read_fits.c) ---- */

static int next_of_kind(int kind)
{
    for (int n = g_cur + 1; n <= g_nhdu + 1; n++)
        if (g_hdu[n - 2].kind == kind) return n;
    return 0;
}

int read_oi_target(fitsfile *fptr, oi_target *targets, int *status)
{
    (void)fptr;
    if (*status) return *status;
    targets->revision = 1;
    targets->ntarget = 1;
    targets->targ = calloc(1, sizeof(target));
    targets->targ[0].target_id = g_target_id;
    strcpy(targets->targ[0].target, g_target_name);
    return 0;
}

int read_oi_wavelength(fitsfile *fptr, char *insname, oi_wavelength *wave, int *status)
{
    (void)fptr;
    if (*status) return *status;
    for (int i = 0; i < g_nhdu; i++) {
        const mem_hdu *h = &g_hdu[i];
        if (h->kind == MEM_WAVE && strcmp(h->insname, insname) == 0) {
            wave->revision = 1;
            strcpy(wave->insname, h->insname);
            wave->nwave = h->nwave;
            wave->eff_wave = dup_mem(h->eff_wave, sizeof(float) * h->nwave);
            wave->eff_band = dup_mem(h->eff_band, sizeof(float) * h->nwave);
            return 0;
        }
    }
    return (*status = END_OF_FILE);
}

int read_next_oi_vis2(fitsfile *fptr, oi_vis2 *vis2, int *status)
{
    (void)fptr;
    if (*status) return *status;
    int n = next_of_kind(MEM_VIS2);
    if (!n) return (*status = END_OF_FILE);
    g_cur = n;
    const mem_hdu *h = &g_hdu[n - 2];
    vis2->revision = 1;
    vis2->date_obs[0] = '\0';
    vis2->arrname[0] = '\0';
    strcpy(vis2->insname, h->insname);
    vis2->numrec = h->numrec;
    vis2->nwave = h->nwave;
    vis2->record = malloc(sizeof(oi_vis2_record) * (h->numrec ? h->numrec : 1));
    for (long r = 0; r < h->numrec; r++) {
        oi_vis2_record *rec = &vis2->record[r];
        memset(rec, 0, sizeof(*rec));
        rec->target_id = h->target_id[r];
        rec->vis2data = dup_mem(h->c0 + r * h->nwave, sizeof(double) * h->nwave);
        rec->vis2err = dup_mem(h->c1 + r * h->nwave, sizeof(double) * h->nwave);
        rec->ucoord = h->u1[r];
        rec->vcoord = h->v1[r];
        rec->flag = dup_mem(h->flag + r * h->nwave, h->nwave);
    }
    return 0;
}

int read_next_oi_t3(fitsfile *fptr, oi_t3 *t3, int *status)
{
    (void)fptr;
    if (*status) return *status;
    int n = next_of_kind(MEM_T3);
    if (!n) return (*status = END_OF_FILE);
    g_cur = n;
    const mem_hdu *h = &g_hdu[n - 2];
    t3->revision = 1;
    t3->date_obs[0] = '\0';
    t3->arrname[0] = '\0';
    strcpy(t3->insname, h->insname);
    t3->numrec = h->numrec;
    t3->nwave = h->nwave;
    t3->record = malloc(sizeof(oi_t3_record) * (h->numrec ? h->numrec : 1));
    for (long r = 0; r < h->numrec; r++) {
        oi_t3_record *rec = &t3->record[r];
        memset(rec, 0, sizeof(*rec));
        rec->target_id = h->target_id[r];
        rec->t3amp = dup_mem(h->c0 + r * h->nwave, sizeof(double) * h->nwave);
        rec->t3amperr = dup_mem(h->c1 + r * h->nwave, sizeof(double) * h->nwave);
        rec->t3phi = dup_mem(h->c2 + r * h->nwave, sizeof(double) * h->nwave);
        rec->t3phierr = dup_mem(h->c3 + r * h->nwave, sizeof(double) * h->nwave);
        rec->u1coord = h->u1[r];
        rec->v1coord = h->v1[r];
        rec->u2coord = h->u2[r];
        rec->v2coord = h->v2[r];
        rec->flag = dup_mem(h->flag + r * h->nwave, h->nwave);
    }
    return 0;
}
