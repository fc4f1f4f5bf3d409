/*
 * oi_index.c -- OIFITS record -> (uv list, triangle references) indexer.
 *
 * Restates get_oi_fits_data (gpair1/trunk/getoifits.c:65-357) with the same
 * output, bit for bit:
 *   * V2 points in table / record / channel order, u = (float)(ucoord/lambda),
 *     folded into u >= 0 (getoifits.c:140-151); every V2 point is a uv point;
 *   * each T3 vertex (uv1, uv2, uv3 = -(uv1+uv2) in float, getoifits.c:209-216)
 *     is matched against the uv points that exist at that moment with
 *     compare_uv (getoifits.c:17-62, threshold 5e-5) AND exact wavelength
 *     equality; the lowest-index match wins and its compare_uv result gives the
 *     sign; unmatched vertices are appended (folded, sign -1 when folded);
 *   * NaN triple amplitudes become amplitude 1 with error 1e99 (getoifits.c:193-197);
 *   * band limits in nm and per-channel flags as in getoifits.c:133-134, 185-187;
 *     a table is used when its first record's TARGET_ID is the selected one.
 *
 * The reference scans all uv points for every vertex (O(nbis * nuv)). Here the
 * points are bucketed by (wavelength bits, log2|u| bucket, log2|v| bucket) and
 * only the 3x3 neighbourhoods of (u, v) and of (-u, -v) are examined, each
 * candidate verified with the reference's own compare_uv arithmetic. A match
 * needs |u2/u1 - 1| < ~7e-5 (and the same for v, or for -u, -v), far inside
 * one bucket (2^(1/64) - 1 = 1.1%), so the minimum matching index is always
 * among the candidates. Coordinates outside the bucketed range (non-finite,
 * |x| >= 1e18 where compare_uv's float squares overflow, so that any query can
 * match) are handled exactly: such stored points are checked for every query,
 * and such queries fall back to the reference's linear scan.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gpair_b200.h"

#define UV_THRESHOLD 5.0e-5
#define BILLION (1.0e9)
#define INF_ERR 1e99

/* compare_uv, gpair1/trunk/getoifits.c:17-62: same float/double mix. */
static int oi_compare_uv(float u1, float v1, float u2, float v2, float thresh)
{
    float sqthresh = thresh * thresh;
    float pcompu = 2.0 * (u1 - u2) * (u1 - u2) / (u1 * u1 + u2 * u2);
    float pcompv = 2.0 * (v1 - v2) * (v1 - v2) / (v1 * v1 + v2 * v2);
    float mcompu = 2.0 * (u1 + u2) * (u1 + u2) / (u1 * u1 + u2 * u2);
    float mcompv = 2.0 * (v1 + v2) * (v1 + v2) / (v1 * v1 + v2 * v2);
    if ((u1 - u2) == 0.0) pcompu = 0.0;
    if ((v1 - v2) == 0.0) pcompv = 0.0;
    if ((u1 + u2) == 0.0) mcompu = 0.0;
    if ((v1 + v2) == 0.0) mcompv = 0.0;
    if ((pcompu < sqthresh) && (pcompv < sqthresh)) return 1;
    if ((mcompu < sqthresh) && (mcompv < sqthresh)) return -1;
    return 0;
}

/* ---------------------------------------------------------------- buckets */

#define TINY_EXP (-60)
static int oi_weird(float x) { return !isfinite(x) || fabsf(x) >= 1e18f; }

/* continuous integer bucket line: 0 = |x| < 2^-60 (incl. 0), +-k for log2 buckets */
static int64_t oi_bucket(float x)
{
    float a = fabsf(x);
    if (a < 0x1p-60f) return 0;
    int64_t b = (int64_t)floor(log2((double)a) * 64.0) - (int64_t)(TINY_EXP * 64) + 1;
    return x < 0 ? -b : b;
}

typedef struct {
    uint64_t key;
    int32_t head; /* first point index in this bucket (ascending chain) */
    int32_t tail;
} oi_slot;

typedef struct {
    oi_slot *slots;
    int64_t cap; /* power of two */
    int64_t used;
    int32_t *next; /* per point: next index in the same bucket */
    int64_t next_cap;
    int32_t *weird; /* stored points with non-bucketable coordinates */
    int64_t nweird, weird_cap;
} oi_hash;

static uint64_t oi_mix(uint64_t k)
{
    k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ULL; k ^= k >> 33;
    return k;
}

static uint64_t oi_key(float w, int64_t bu, int64_t bv)
{
    uint32_t wb;
    if (w == 0.0f) w = 0.0f; /* -0 == +0 */
    memcpy(&wb, &w, 4);
    return ((uint64_t)wb << 32) ^ ((uint64_t)(bu & 0xffff) << 16) ^ (uint64_t)(bv & 0xffff)
           ^ ((uint64_t)(bu >> 16) * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)(bv >> 16) * 0xC2B2AE3D27D4EB4FULL);
}

static int oi_hash_grow(oi_hash *h)
{
    int64_t ncap = h->cap ? h->cap * 2 : 1024;
    oi_slot *ns = malloc(sizeof(oi_slot) * ncap);
    if (!ns) return -1;
    for (int64_t i = 0; i < ncap; i++) ns[i].head = -1;
    for (int64_t i = 0; i < h->cap; i++) {
        if (h->slots[i].head < 0) continue;
        uint64_t p = oi_mix(h->slots[i].key) & (ncap - 1);
        while (ns[p].head >= 0) p = (p + 1) & (ncap - 1);
        ns[p] = h->slots[i];
    }
    free(h->slots);
    h->slots = ns;
    h->cap = ncap;
    return 0;
}

/* exact key match requires storing (w, bu, bv); we keep the hashed key and
 * re-verify candidates with compare_uv, so key collisions only add candidates. */
static oi_slot *oi_find(oi_hash *h, uint64_t key)
{
    if (!h->cap) return NULL;
    uint64_t p = oi_mix(key) & (h->cap - 1);
    while (h->slots[p].head >= 0) {
        if (h->slots[p].key == key) return &h->slots[p];
        p = (p + 1) & (h->cap - 1);
    }
    return NULL;
}

static int oi_insert(oi_hash *h, const gpair_uv *uv, int32_t idx)
{
    if (idx >= h->next_cap) {
        int64_t nc = h->next_cap ? h->next_cap * 2 : 4096;
        while (nc <= idx) nc *= 2;
        int32_t *nn = realloc(h->next, sizeof(int32_t) * nc);
        if (!nn) return -1;
        h->next = nn;
        h->next_cap = nc;
    }
    h->next[idx] = -1;
    const gpair_uv *p = &uv[idx];
    if (oi_weird(p->u) || oi_weird(p->v) || isnan(p->wavelength)) {
        if (h->nweird == h->weird_cap) {
            int64_t nc = h->weird_cap ? h->weird_cap * 2 : 16;
            int32_t *nw = realloc(h->weird, sizeof(int32_t) * nc);
            if (!nw) return -1;
            h->weird = nw;
            h->weird_cap = nc;
        }
        h->weird[h->nweird++] = idx;
        return 0;
    }
    uint64_t key = oi_key(p->wavelength, oi_bucket(p->u), oi_bucket(p->v));
    oi_slot *s = oi_find(h, key);
    if (s) {
        h->next[s->tail] = idx;
        s->tail = idx;
        return 0;
    }
    if ((h->used + 1) * 2 > h->cap && oi_hash_grow(h)) return -1;
    uint64_t q = oi_mix(key) & (h->cap - 1);
    while (h->slots[q].head >= 0) q = (q + 1) & (h->cap - 1);
    h->slots[q].key = key;
    h->slots[q].head = idx;
    h->slots[q].tail = idx;
    h->used++;
    return 0;
}

static void oi_hash_free(oi_hash *h)
{
    free(h->slots); free(h->next); free(h->weird);
    memset(h, 0, sizeof(*h));
}

/* Lowest-index uv point matching (u, v) at wavelength w; returns -1 if none,
 * else the index, with *sign = compare_uv result. */
static int64_t oi_match(const oi_hash *h, const gpair_uv *uv, int64_t nuv, float u, float v, float w, int *sign)
{
    int64_t best = -1;
    int bsign = 0;
    if (oi_weird(u) || oi_weird(v)) {
        for (int64_t l = 0; l < nuv; l++) {
            int npve = oi_compare_uv(u, v, uv[l].u, uv[l].v, UV_THRESHOLD);
            if (npve != 0 && w == uv[l].wavelength) { *sign = npve; return l; }
        }
        return -1;
    }
    for (int64_t i = 0; i < h->nweird; i++) {
        int32_t l = h->weird[i];
        int npve = oi_compare_uv(u, v, uv[l].u, uv[l].v, UV_THRESHOLD);
        if (npve != 0 && w == uv[l].wavelength && (best < 0 || l < best)) { best = l; bsign = npve; }
    }
    if (!isnan(w)) {
        int64_t bu[2] = {oi_bucket(u), oi_bucket(-u)}, bv[2] = {oi_bucket(v), oi_bucket(-v)};
        for (int side = 0; side < 2; side++)
            for (int du = -1; du <= 1; du++)
                for (int dv = -1; dv <= 1; dv++) {
                    const oi_slot *s = oi_find((oi_hash *)h, oi_key(w, bu[side] + du, bv[side] + dv));
                    if (!s) continue;
                    for (int32_t l = s->head; l >= 0; l = h->next[l]) {
                        if (best >= 0 && l >= best) break; /* chains are ascending */
                        int npve = oi_compare_uv(u, v, uv[l].u, uv[l].v, UV_THRESHOLD);
                        if (npve != 0 && w == uv[l].wavelength) { best = l; bsign = npve; break; }
                    }
                }
    }
    if (best >= 0) *sign = bsign;
    return best;
}

/* ------------------------------------------------------------------ driver */

typedef struct {
    gpair_oi_data *d;
    int64_t cap_pow, cap_bis, cap_uv;
} oi_out;

static int oi_reserve(void **p, int64_t *cap, int64_t need, size_t elt)
{
    if (need <= *cap) return 0;
    int64_t nc = *cap ? *cap : 1024;
    while (nc < need) nc *= 2;
    void *np = realloc(*p, elt * nc);
    if (!np) return -1;
    *p = np;
    *cap = nc;
    return 0;
}

static const gpair_oi_wavelength *oi_find_wave(int nw, const gpair_oi_wavelength *w, const char *insname)
{
    for (int i = 0; i < nw; i++)
        if (strcmp(w[i].insname, insname) == 0) return &w[i];
    return NULL;
}

void gpair_free_oi_data(gpair_oi_data *d)
{
    if (!d) return;
    free(d->pow); free(d->powerr); free(d->bisamp); free(d->bisamperr); free(d->bisphs); free(d->bisphserr);
    free(d->uv); free(d->uvpnt); free(d->sign);
    memset(d, 0, sizeof(*d));
}

int gpair_get_oi_fits_data(int target_id, float minband, float maxband, int nwave_tables,
                           const gpair_oi_wavelength *waves, int nvis2_tables, const gpair_oi_vis2 *vis2,
                           int nt3_tables, const gpair_oi_t3 *t3, gpair_oi_data *out)
{
    if (!out) return GPAIR_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    int64_t cap_pow = 0, cap_pe = 0, cap_bis[4] = {0, 0, 0, 0}, cap_uv = 0, cap_ref = 0, cap_sign = 0;
    oi_hash h;
    memset(&h, 0, sizeof(h));
    int rc = GPAIR_OK;

    for (int t = 0; t < nvis2_tables; t++) {
        const gpair_oi_vis2 *tb = &vis2[t];
        const gpair_oi_wavelength *wave = oi_find_wave(nwave_tables, waves, tb->insname);
        if (!wave) break; /* the reference's read loop ends when a wavelength lookup fails */
        if (tb->numrec <= 0 || tb->target_id[0] != target_id) continue;
        for (long i = 0; i < tb->numrec; i++) {
            for (int k = 0; k < tb->nwave; k++) {
                size_t c = (size_t)i * tb->nwave + k;
                if (((wave->eff_wave[k] * BILLION) > minband) && ((wave->eff_wave[k] * BILLION) < maxband)
                    && (!(tb->flag[c]))) {
                    int64_t np = out->npow, nu = out->nuv;
                    if (oi_reserve((void **)&out->pow, &cap_pow, np + 1, sizeof(float))
                        || oi_reserve((void **)&out->powerr, &cap_pe, np + 1, sizeof(float))
                        || oi_reserve((void **)&out->uv, &cap_uv, nu + 1, sizeof(gpair_uv))) { rc = GPAIR_ERR_ALLOC; goto done; }
                    out->pow[np] = (float)tb->vis2data[c];
                    out->powerr[np] = (float)tb->vis2err[c];
                    gpair_uv *p = &out->uv[nu];
                    p->u = (float)(tb->ucoord[i] / wave->eff_wave[k]);
                    p->v = (float)(tb->vcoord[i] / wave->eff_wave[k]);
                    p->wavelength = wave->eff_wave[k];
                    p->bandwidth = wave->eff_band[k];
                    if (p->u < 0.0) { p->u = -p->u; p->v = -p->v; }
                    if (oi_insert(&h, out->uv, (int32_t)nu)) { rc = GPAIR_ERR_ALLOC; goto done; }
                    out->npow++;
                    out->nuv++;
                }
            }
        }
    }

    for (int t = 0; t < nt3_tables; t++) {
        const gpair_oi_t3 *tb = &t3[t];
        const gpair_oi_wavelength *wave = oi_find_wave(nwave_tables, waves, tb->insname);
        if (!wave) break;
        if (tb->numrec <= 0 || tb->target_id[0] != target_id) continue;
        for (long i = 0; i < tb->numrec; i++) {
            for (int k = 0; k < tb->nwave; k++) {
                size_t c = (size_t)i * tb->nwave + k;
                if (!(((wave->eff_wave[k] * BILLION) > minband) && ((wave->eff_wave[k] * BILLION) < maxband)
                      && (!(tb->flag[c]))))
                    continue;
                int64_t nb = out->nbis;
                if (oi_reserve((void **)&out->bisamp, &cap_bis[0], nb + 1, sizeof(float))
                    || oi_reserve((void **)&out->bisamperr, &cap_bis[1], nb + 1, sizeof(float))
                    || oi_reserve((void **)&out->bisphs, &cap_bis[2], nb + 1, sizeof(float))
                    || oi_reserve((void **)&out->bisphserr, &cap_bis[3], nb + 1, sizeof(float))
                    || oi_reserve((void **)&out->uvpnt, &cap_ref, 3 * (nb + 1), sizeof(int64_t))
                    || oi_reserve((void **)&out->sign, &cap_sign, 3 * (nb + 1), sizeof(int16_t))) { rc = GPAIR_ERR_ALLOC; goto done; }
                if (isnan(tb->t3amp[c])) {
                    out->bisamp[nb] = 1.0;
                    out->bisamperr[nb] = INF_ERR;
                } else {
                    out->bisamp[nb] = (float)tb->t3amp[c];
                    out->bisamperr[nb] = (float)tb->t3amperr[c];
                }
                out->bisphs[nb] = (float)tb->t3phi[c];
                out->bisphserr[nb] = (float)tb->t3phierr[c];
                float pu[3], pv[3];
                pu[0] = (float)(tb->u1coord[i] / wave->eff_wave[k]);
                pv[0] = (float)(tb->v1coord[i] / wave->eff_wave[k]);
                pu[1] = (float)(tb->u2coord[i] / wave->eff_wave[k]);
                pv[1] = (float)(tb->v2coord[i] / wave->eff_wave[k]);
                pu[2] = -(pu[0] + pu[1]);
                pv[2] = -(pv[0] + pv[1]);
                float w = wave->eff_wave[k];
                for (int vtx = 0; vtx < 3; vtx++) {
                    int sgn = 1;
                    int64_t l = oi_match(&h, out->uv, out->nuv, pu[vtx], pv[vtx], w, &sgn);
                    if (l >= 0) {
                        out->uvpnt[3 * nb + vtx] = l;
                        out->sign[3 * nb + vtx] = (int16_t)sgn;
                    } else {
                        int64_t nu = out->nuv;
                        if (oi_reserve((void **)&out->uv, &cap_uv, nu + 1, sizeof(gpair_uv))) { rc = GPAIR_ERR_ALLOC; goto done; }
                        gpair_uv *p = &out->uv[nu];
                        p->u = pu[vtx];
                        p->v = pv[vtx];
                        p->wavelength = w;
                        p->bandwidth = wave->eff_band[k];
                        out->uvpnt[3 * nb + vtx] = nu;
                        out->sign[3 * nb + vtx] = 1;
                        if (p->u < 0.0) {
                            p->u = -pu[vtx];
                            p->v = -pv[vtx];
                            out->sign[3 * nb + vtx] = -1;
                        }
                        if (oi_insert(&h, out->uv, (int32_t)nu)) { rc = GPAIR_ERR_ALLOC; goto done; }
                        out->nuv++;
                    }
                }
                out->nbis++;
            }
        }
    }
done:
    oi_hash_free(&h);
    if (rc != GPAIR_OK) gpair_free_oi_data(out);
    return rc;
}
