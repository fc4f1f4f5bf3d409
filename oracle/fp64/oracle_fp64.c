/*
 * oracle_fp64.c -- CPU oracle for the GPAIR reconstruction hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (gpair_b200/, include/)
 * links or calls this file; tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it as the checker. It restates the reference's
 * algorithm in FP64 (plus exact-float replicas of its host-side setup):
 *
 *   o_init_data          gpair1/trunk/gpair.c:997-1066 (float, bit-exact replica)
 *   o_dft_tables_f32     gpair1/trunk/gpair.c:231-245 (float tables, reference formula)
 *   o64_image2vis        gpair1/trunk/cpu.c:449-475 (FP64 twiddles from the same phase)
 *   o64_vis2data         gpair1/trunk/cpu.c:758-802
 *   o64_data2chi2        gpair1/trunk/cpu.c:371-383
 *   o64_entropy(_grad)   gpair1/trunk/cpu.c:385-412 (gradient keeps the previous
 *                        value where image <= 0 or model <= 0)
 *   o64_data_gradient    gpair1/trunk/cpu.c:279-369 (direct per-pixel sum)
 *   o64_cg_run           gpair1/trunk/gpair.c:682-915 + gpair1/trunk/gpu.c:1947-2065
 *   o32_ref_cg_run       the same CG in float, evaluating with the reference's
 *                        own compiled cpu.c (oracle/_ref/libgpair_ref.so), which
 *                        the caller passes in as function pointers
 *
 * Parity of the restatement is pinned in tests against the reference's own
 * compiled cpu.c and getoifits.c (oracle/_ref) on seeded synthetic problems
 * and on the reference's OIFITS fixture.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O_PI 3.14159265358979323
#define O_RPMAS ((3.14159265358979323 / 180.0) / 3600000.0)

static float o_square(float x) { return x * x; }

/* ------------------------------------------------------------------ setup */

/* Data packing, gpair1/trunk/gpair.c:997-1066. bisamp/bisamperr are updated in
 * place when triple amplitudes are extrapolated, as the reference does.
 * Returns the change to ndof (minus one per failed extrapolation). */
int o_init_data(int do_extrapolation, int npow, int nbis, const float *pow, const float *powerr,
                float *bisamp, float *bisamperr, const float *bisphs, const float *bisphserr,
                const int64_t *uvpnt, float *data, float *data_err, float *phasor /* complex64 */)
{
    int ndof_delta = 0;
    float complex *ph = (float complex *)phasor;
    for (int ii = 0; ii < npow; ii++) {
        data[ii] = pow[ii];
        data_err[ii] = 1. / fabs(powerr[ii]);
    }
    for (int ii = 0; ii < nbis; ii++) {
        if ((do_extrapolation == 1) && ((bisamperr[ii] <= 0.) || (bisamperr[ii] > 1e3))) {
            int64_t a = uvpnt[3 * ii], b = uvpnt[3 * ii + 1], c = uvpnt[3 * ii + 2];
            if ((a < npow) && (b < npow) && (c < npow)) {
                float pow1 = pow[a], powerr1 = powerr[a];
                float pow2 = pow[b], powerr2 = powerr[b];
                float pow3 = pow[c], powerr3 = powerr[c];
                float sqamp1 = (pow1 + sqrt(o_square(pow1) + 2.0 * o_square(powerr1))) / 2.;
                float sqamperr1 = 1. / (1. / sqamp1 + 2. * (3. * sqamp1 - pow1) / o_square(powerr1));
                float sqamp2 = (pow2 + sqrt(o_square(pow2) + 2.0 * o_square(powerr2))) / 2.;
                float sqamperr2 = 1. / (1. / sqamp2 + 2. * (3. * sqamp2 - pow2) / o_square(powerr2));
                float sqamp3 = (pow3 + sqrt(o_square(pow3) + 2.0 * o_square(powerr3))) / 2.;
                float sqamperr3 = 1. / (1. / sqamp3 + 2. * (3. * sqamp3 - pow3) / o_square(powerr3));
                bisamp[ii] = sqrt(sqamp1 * sqamp2 * sqamp3);
                bisamperr[ii] = bisamp[ii] * sqrt(sqamperr1 / sqamp1 + sqamperr2 / sqamp2 + sqamperr3 / sqamp3);
            } else {
                bisamp[ii] = 1.0;
                bisamperr[ii] = 1e99;
                ndof_delta--;
            }
        }
        data[npow + 2 * ii] = fabs(bisamp[ii]);
        data[npow + 2 * ii + 1] = 0.;
        data_err[npow + 2 * ii] = 1. / bisamperr[ii];
        data_err[npow + 2 * ii + 1] = 1. / fabs(bisamp[ii] * bisphserr[ii] * O_PI / 180.);
        ph[ii] = cexp(-I * bisphs[ii] * O_PI / 180.);
    }
    return ndof_delta;
}

/* Float DFT tables in the CPU layout [nuv][N], gpair1/trunk/gpair.c:231-245:
 * the phase is formed in double exactly as the reference's expression orders
 * it, then exponentiated and rounded to complex64. */
void o_dft_tables_f32(int N, int nuv, const float *uv /* [nuv][4] */, float pix, float *dftx, float *dfty)
{
    float complex *tx = (float complex *)dftx, *ty = (float complex *)dfty;
    for (int uu = 0; uu < nuv; uu++) {
        float u = uv[4 * uu], v = uv[4 * uu + 1];
        for (int ii = 0; ii < N; ii++) {
            tx[N * uu + ii] = cexp(2.0 * I * O_PI * (3.14159265358979323 / 180.0) / 3600000.0 * pix * u * (float)ii);
            ty[N * uu + ii] = cexp(-2.0 * I * O_PI * (3.14159265358979323 / 180.0) / 3600000.0 * pix * v * (float)ii);
        }
    }
}

/* FP64 twiddle phase (radians) for coordinate `w` (u or v, in wavelengths) at
 * pixel index `i`, same factor ordering as the reference's table build. */
static inline double o64_phase(float pix, float w, int i)
{
    return (((2.0 * O_PI) * (3.14159265358979323 / 180.0)) / 3600000.0) * (double)pix * (double)w * (double)(float)i;
}

/* --------------------------------------------------------------- forward */

/* V_k = sum_{y,x} I[y*N+x] e^{+i phase(u_k,x)} e^{-i phase(v_k,y)} / F,
 * divided by F only when F > 0 (gpair1/trunk/cpu.c:449-475). */
void o64_image2vis(int N, int nuv, const double *image, const float *uv, float pix, double *visi /* c128 */)
{
    double complex *V = (double complex *)visi;
    double F = 0;
    for (int i = 0; i < N * N; i++) F += image[i];
    double complex *ex = malloc(sizeof(double complex) * N), *ey = malloc(sizeof(double complex) * N);
    for (int k = 0; k < nuv; k++) {
        for (int i = 0; i < N; i++) {
            double px = o64_phase(pix, uv[4 * k], i), py = o64_phase(pix, uv[4 * k + 1], i);
            ex[i] = cos(px) + I * sin(px);
            ey[i] = cos(py) - I * sin(py);
        }
        double complex acc = 0;
        for (int y = 0; y < N; y++) {
            double complex row = 0;
            for (int x = 0; x < N; x++) row += image[y * N + x] * ex[x];
            acc += row * ey[y];
        }
        V[k] = (F > 0.) ? acc / F : acc;
    }
    free(ex); free(ey);
}

/* mock[k] = |V_k|^2 (k < npow); T3 = V~ab V~bc V~ca phasor (gpair1/trunk/cpu.c:758-802) */
void o64_vis2data(int npow, int nbis, const double *visi, const double *phasor /* c128 */,
                  const int64_t *uvpnt, const int16_t *sign, double *mock)
{
    const double complex *V = (const double complex *)visi, *ph = (const double complex *)phasor;
    for (int i = 0; i < npow; i++) {
        double a = cabs(V[i]);
        mock[i] = a * a;
    }
    for (int t = 0; t < nbis; t++) {
        double complex vab = V[uvpnt[3 * t]], vbc = V[uvpnt[3 * t + 1]], vca = V[uvpnt[3 * t + 2]];
        if (sign[3 * t] < 0) vab = conj(vab);
        if (sign[3 * t + 1] < 0) vbc = conj(vbc);
        if (sign[3 * t + 2] < 0) vca = conj(vca);
        double complex t3 = (vab * vbc * vca) * ph[t];
        mock[npow + 2 * t] = creal(t3);
        mock[npow + 2 * t + 1] = cimag(t3);
    }
}

double o64_data2chi2(int ndata, const float *data, const float *data_err, const double *mock)
{
    double chi2 = 0;
    for (int i = 0; i < ndata; i++) {
        double t = (mock[i] - data[i]) * data_err[i];
        chi2 += t * t;
    }
    return chi2;
}

double o64_entropy(int npix, const double *image, const float *model)
{
    double S = 0;
    for (int i = 0; i < npix; i++) {
        if (image[i] > 0. && model[i] > 0.) S += image[i] - model[i] - image[i] * log(image[i] / model[i]);
        else S += -model[i];
    }
    return S;
}

/* Where image <= 0 or model <= 0 the previous gradient value is kept. */
void o64_entropy_gradient(int npix, const double *image, const float *model, double *grad)
{
    for (int i = 0; i < npix; i++)
        if (image[i] > 0. && model[i] > 0.) grad[i] = -log(image[i] / model[i]);
}

/* d chi2 / d I(x,y), direct per-pixel sum over every V2 point and triangle
 * (gpair1/trunk/cpu.c:279-369), with FP64 twiddles. Uses visi/mock of the
 * same image. grad is [N*N] with x fastest. Rows are shared out over
 * `o_threads` pthreads (the sum per pixel is unchanged). */
typedef struct {
    int N, npow, nbis;
    double invflux;
    const float *data, *data_err;
    const double complex *V, *ph, *ex, *ey;
    const int64_t *uvpnt;
    const int16_t *sign;
    const double *mock;
    double *grad;
    int row0, row1;
} o64_grad_job;

static void *o64_grad_rows(void *arg)
{
    o64_grad_job *j = arg;
    const int N = j->N;
    for (int jj = j->row0; jj < j->row1; jj++) {
        for (int ii = 0; ii < N; ii++) {
            double g = 0;
            for (int k = 0; k < j->npow; k++) {
                double complex e = j->ex[(size_t)k * N + ii] * j->ey[(size_t)k * N + jj];
                g += 4.0 * (double)j->data_err[k] * j->data_err[k] * j->invflux * (j->mock[k] - j->data[k])
                     * creal(conj(j->V[k]) * (e - j->V[k]));
            }
            for (int t = 0; t < j->nbis; t++) {
                int64_t a = j->uvpnt[3 * t], b = j->uvpnt[3 * t + 1], c = j->uvpnt[3 * t + 2];
                double complex vab = j->V[a], vbc = j->V[b], vca = j->V[c];
                double complex dab = j->ex[(size_t)a * N + ii] * j->ey[(size_t)a * N + jj];
                double complex dbc = j->ex[(size_t)b * N + ii] * j->ey[(size_t)b * N + jj];
                double complex dca = j->ex[(size_t)c * N + ii] * j->ey[(size_t)c * N + jj];
                if (j->sign[3 * t] < 0) { vab = conj(vab); dab = conj(dab); }
                if (j->sign[3 * t + 1] < 0) { vbc = conj(vbc); dbc = conj(dbc); }
                if (j->sign[3 * t + 2] < 0) { vca = conj(vca); dca = conj(dca); }
                double complex t3der = ((dab - vab) * vbc * vca + vab * (dbc - vbc) * vca + vab * vbc * (dca - vca))
                                       * j->ph[t] * j->invflux;
                int r = j->npow + 2 * t;
                g += 2. * (double)j->data_err[r] * j->data_err[r] * (j->mock[r] - j->data[r]) * creal(t3der);
                g += 2. * (double)j->data_err[r + 1] * j->data_err[r + 1] * j->mock[r + 1] * cimag(t3der);
            }
            j->grad[ii + jj * N] = g;
        }
    }
    return NULL;
}

int o_threads = 8;

void o_set_threads(int n) { o_threads = n < 1 ? 1 : n; }

void o64_data_gradient(int N, int npow, int nbis, const double *image, const float *uv, float pix,
                       const float *data, const float *data_err, const double *phasor,
                       const int64_t *uvpnt, const int16_t *sign, const double *visi, const double *mock,
                       double *grad)
{
    double flux = 0;
    for (int i = 0; i < N * N; i++) flux += image[i];
    int nuv_used = npow;
    for (int t = 0; t < 3 * nbis; t++) if (uvpnt[t] + 1 > nuv_used) nuv_used = (int)uvpnt[t] + 1;
    double complex *ex = malloc(sizeof(double complex) * (size_t)(nuv_used ? nuv_used : 1) * N);
    double complex *ey = malloc(sizeof(double complex) * (size_t)(nuv_used ? nuv_used : 1) * N);
    for (int k = 0; k < nuv_used; k++)
        for (int i = 0; i < N; i++) {
            double px = o64_phase(pix, uv[4 * k], i), py = o64_phase(pix, uv[4 * k + 1], i);
            ex[(size_t)k * N + i] = cos(px) + I * sin(px);
            ey[(size_t)k * N + i] = cos(py) - I * sin(py);
        }
    int nt = o_threads > N ? N : o_threads;
    pthread_t th[64];
    o64_grad_job jobs[64];
    if (nt > 64) nt = 64;
    for (int t = 0; t < nt; t++) {
        o64_grad_job jb = {N, npow, nbis, 1. / flux, data, data_err, (const double complex *)visi,
                           (const double complex *)phasor, ex, ey, uvpnt, sign, mock, grad,
                           (int)((long)N * t / nt), (int)((long)N * (t + 1) / nt)};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, o64_grad_rows, &jobs[t]);
    }
    for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
    free(ex); free(ey);
}

/* ------------------------------------------------------------------- CG */

#define REAL double
#define CG(name) o64_##name
#include "cg_impl.h"
#undef REAL
#undef CG

#define REAL float
#define CG(name) o32_##name
#include "cg_impl.h"
#undef REAL
#undef CG

/* The projected L-BFGS direction of the batched search (two-loop recursion)
 * for caller-given pairs: S and Y hold `count` pairs of n values, oldest
 * first, of which the newest LBFGS_PAIRS are used, as in the search; gamma
 * scales the initial matrix. Lets the tests check other formulations of the
 * same direction against this one. */
void o64_lbfgs_direction(int n, int count, const double *S, const double *Y, double gamma, const double *image,
                         const double *g, double minvalue, double *d)
{
    o64_lbfgs L;
    memset(&L, 0, sizeof(L));
    const int use = count < LBFGS_PAIRS ? count : LBFGS_PAIRS;
    L.s = (double *)S + (size_t)(count - use) * n;
    L.y = (double *)Y + (size_t)(count - use) * n;
    L.gamma = gamma;
    L.count = use;
    L.head = use;  /* newest pair in slot use - 1 */
    for (int j = 0; j < use; j++) {
        double sy = 0;
        for (int i = 0; i < n; i++) sy += L.s[(size_t)j * n + i] * L.y[(size_t)j * n + i];
        L.rho[j] = 1.0 / sy;
    }
    o64_lbfgs_dir(&L, n, image, g, minvalue, d);
}

/* FP64 evaluator over a problem: chi2 (image2vis + vis2data + data2chi2),
 * Gull-Skilling entropy, and gradient = d chi2 - alpha * dS with the
 * entropy-gradient buffer persisting between calls. */
typedef struct {
    int N, nuv, npow, nbis;
    const float *uv;
    float pix;
    const float *data, *data_err;
    const double *phasor;
    const int64_t *uvpnt;
    const int16_t *sign;
    const float *model;
    double alpha;
    double *visi, *mock, *egrad, *dgrad;
} o64_problem;

static double o64_eval_criterion(void *ctx, const double *image, double *chi2, double *S)
{
    o64_problem *p = ctx;
    o64_image2vis(p->N, p->nuv, image, p->uv, p->pix, p->visi);
    o64_vis2data(p->npow, p->nbis, p->visi, p->phasor, p->uvpnt, p->sign, p->mock);
    *chi2 = o64_data2chi2(p->npow + 2 * p->nbis, p->data, p->data_err, p->mock);
    *S = o64_entropy(p->N * p->N, image, p->model);
    return *chi2 - p->alpha * *S;
}

static void o64_eval_gradient(void *ctx, const double *image, double *grad)
{
    o64_problem *p = ctx;
    int n = p->N * p->N;
    o64_data_gradient(p->N, p->npow, p->nbis, image, p->uv, p->pix, p->data, p->data_err, p->phasor,
                      p->uvpnt, p->sign, p->visi, p->mock, p->dgrad);
    o64_entropy_gradient(n, image, p->model, p->egrad);
    for (int i = 0; i < n; i++) grad[i] = p->dgrad[i] - p->alpha * p->egrad[i];
}

/* Full FP64 reconstruction: `iterations` CG iterations from `image`, with the
 * reference's line search (line_search 0) or the batched search (1).
 * trace arrays (length iterations) may be NULL. Returns 0 on success. */
int o64_reconstruct(int N, int nuv, int npow, int nbis, const float *uv, float pix, const float *data,
                    const float *data_err, const float *phasor_c64, const int64_t *uvpnt, const int16_t *sign,
                    const float *model, double alpha, int method, int iterations, double *image,
                    int *criterion_evals, int *grad_evals, double *J, double *chi2, double *entropy,
                    double *step, double *beta, int line_search, double batch_step_max)
{
    o64_problem p = {N, nuv, npow, nbis, uv, pix, data, data_err, NULL, uvpnt, sign, model, alpha};
    double *ph = malloc(sizeof(double) * 2 * (nbis ? nbis : 1));
    for (int i = 0; i < 2 * nbis; i++) ph[i] = phasor_c64[i];
    p.phasor = ph;
    p.visi = calloc(2 * (size_t)nuv, sizeof(double));
    p.mock = calloc(npow + 2 * (size_t)nbis + 1, sizeof(double));
    p.egrad = calloc((size_t)N * N, sizeof(double));
    p.dgrad = calloc((size_t)N * N, sizeof(double));
    o64_evaluator ev = {&p, o64_eval_criterion, o64_eval_gradient};
    /* c2 = 0.1 is the reference's; projected L-BFGS (method 4, no reference
     * counterpart) uses the usual quasi-Newton curvature constant 0.9 */
    o64_params prm = {method, iterations, 1e-8, 1e-4, method == 4 ? 0.9 : 0.1, 100., 200};
    o64_trace tr = {0, 0, J, chi2, entropy, step, beta};
    int rc = line_search == 1 ? o64_run_batch(&ev, &prm, N * N, image, &tr, batch_step_max)
                              : o64_run(&ev, &prm, N * N, image, &tr);
    *criterion_evals = tr.criterion_evals;
    *grad_evals = tr.grad_evals;
    free(ph); free(p.visi); free(p.mock); free(p.egrad); free(p.dgrad);
    return rc;
}

/* One FP64 criterion + gradient evaluation (chi2, S, visi, mock, data grad). */
double o64_evaluate(int N, int nuv, int npow, int nbis, const float *uv, float pix, const float *data,
                    const float *data_err, const float *phasor_c64, const int64_t *uvpnt, const int16_t *sign,
                    const float *model, const double *image, double *visi, double *mock, double *S,
                    double *data_grad /* may be NULL */)
{
    double *ph = malloc(sizeof(double) * 2 * (nbis ? nbis : 1));
    for (int i = 0; i < 2 * nbis; i++) ph[i] = phasor_c64[i];
    o64_image2vis(N, nuv, image, uv, pix, visi);
    o64_vis2data(npow, nbis, visi, ph, uvpnt, sign, mock);
    double chi2 = o64_data2chi2(npow + 2 * nbis, data, data_err, mock);
    *S = o64_entropy(N * N, image, model);
    if (data_grad)
        o64_data_gradient(N, npow, nbis, image, uv, pix, data, data_err, ph, uvpnt, sign, visi, mock, data_grad);
    free(ph);
    return chi2;
}

/* ------------------------------------------- float CG over the reference */

/* The reference's own compiled functions, passed in by the caller (the
 * oracle does not link oracle/_ref itself). */
typedef float (*o_ref_image2chi2_fn)(const void *problem, float *image, float *visi, float *mock, int quiet);
typedef void (*o_ref_grad_fn)(const void *problem, float *image, float *visi, float *mock, float *grad);
typedef float (*o_ref_entropy_fn)(int N, float *image, float *model);
typedef void (*o_ref_egrad_fn)(int N, float *image, float *model, float *grad);

typedef struct {
    const void *problem;
    int N;
    float *model;
    float alpha;
    o_ref_image2chi2_fn image2chi2;
    o_ref_grad_fn data_gradient;
    o_ref_entropy_fn entropy;
    o_ref_egrad_fn entropy_gradient;
    float *visi, *mock, *dgrad, *egrad;
} o32_refctx;

static float o32_ref_criterion(void *ctx, const float *image, float *chi2, float *S)
{
    o32_refctx *c = ctx;
    *chi2 = c->image2chi2(c->problem, (float *)image, c->visi, c->mock, 1);
    *S = c->entropy(c->N, (float *)image, c->model);
    return *chi2 - c->alpha * *S;
}

static void o32_ref_gradient(void *ctx, const float *image, float *grad)
{
    o32_refctx *c = ctx;
    int n = c->N * c->N;
    c->data_gradient(c->problem, (float *)image, c->visi, c->mock, c->dgrad);
    c->entropy_gradient(c->N, (float *)image, c->model, c->egrad);
    for (int i = 0; i < n; i++) grad[i] = c->dgrad[i] - c->alpha * c->egrad[i];
}

/* Float CG (reference GPU-path control flow) whose criterion and gradient are
 * the reference's own cpu.c functions. This is the CPU baseline that bench.py
 * times. */
int o32_ref_cg_run(const void *problem, int N, int nuv, int ndata, float *model, float alpha, int method,
                   int iterations, float *image, o_ref_image2chi2_fn f_chi2, o_ref_grad_fn f_grad,
                   o_ref_entropy_fn f_ent, o_ref_egrad_fn f_egrad, int *criterion_evals, int *grad_evals,
                   float *J, float *chi2, float *entropy, float *step, float *beta)
{
    o32_refctx c = {problem, N, model, alpha, f_chi2, f_grad, f_ent, f_egrad};
    c.visi = calloc(2 * (size_t)nuv + 2, sizeof(float));
    c.mock = calloc((size_t)ndata + 1, sizeof(float));
    c.dgrad = calloc((size_t)N * N, sizeof(float));
    c.egrad = calloc((size_t)N * N, sizeof(float));
    o32_evaluator ev = {&c, o32_ref_criterion, o32_ref_gradient};
    o32_params prm = {method, iterations, 1e-8f, 1e-4f, 0.1f, 100.f, 200};
    o32_trace tr = {0, 0, J, chi2, entropy, step, beta};
    int rc = o32_run(&ev, &prm, N * N, image, &tr);
    *criterion_evals = tr.criterion_evals;
    *grad_evals = tr.grad_evals;
    free(c.visi); free(c.mock); free(c.dgrad); free(c.egrad);
    return rc;
}

/* The direct gradient (gpair1/trunk/cpu.c:303-368) at selected pixels only,
 * for checks at sizes where the full O(N^2 (npow + nbis)) sum is too slow.
 * pix_x/pix_y hold npx pixel coordinates; grad receives npx values. */
void o64_data_gradient_pixels(int N, int npow, int nbis, int nuv, const double *image, const float *uv, float pix,
                              const float *data, const float *data_err, const float *phasor_c64,
                              const int64_t *uvpnt, const int16_t *sign, const double *visi, const double *mock,
                              int npx, const int *pix_x, const int *pix_y, double *grad)
{
    const double complex *V = (const double complex *)visi;
    double flux = 0;
    for (int i = 0; i < N * N; i++) flux += image[i];
    const double invflux = 1. / flux;
    double complex *ex = malloc(sizeof(double complex) * (nuv ? nuv : 1));
    double complex *ey = malloc(sizeof(double complex) * (nuv ? nuv : 1));
    for (int q = 0; q < npx; q++) {
        const int ii = pix_x[q], jj = pix_y[q];
        for (int k = 0; k < nuv; k++) {
            double px = o64_phase(pix, uv[4 * k], ii), py = o64_phase(pix, uv[4 * k + 1], jj);
            ex[k] = cos(px) + I * sin(px);
            ey[k] = cos(py) - I * sin(py);
        }
        double g = 0;
        for (int k = 0; k < npow; k++) {
            double complex e = ex[k] * ey[k];
            g += 4.0 * (double)data_err[k] * data_err[k] * invflux * (mock[k] - data[k]) * creal(conj(V[k]) * (e - V[k]));
        }
        for (int t = 0; t < nbis; t++) {
            int64_t a = uvpnt[3 * t], b = uvpnt[3 * t + 1], c = uvpnt[3 * t + 2];
            double complex vab = V[a], vbc = V[b], vca = V[c];
            double complex dab = ex[a] * ey[a], dbc = ex[b] * ey[b], dca = ex[c] * ey[c];
            if (sign[3 * t] < 0) { vab = conj(vab); dab = conj(dab); }
            if (sign[3 * t + 1] < 0) { vbc = conj(vbc); dbc = conj(dbc); }
            if (sign[3 * t + 2] < 0) { vca = conj(vca); dca = conj(dca); }
            double complex ph = phasor_c64[2 * t] + I * phasor_c64[2 * t + 1];
            double complex t3der = ((dab - vab) * vbc * vca + vab * (dbc - vbc) * vca + vab * vbc * (dca - vca)) * ph * invflux;
            int r = npow + 2 * t;
            g += 2. * (double)data_err[r] * data_err[r] * (mock[r] - data[r]) * creal(t3der);
            g += 2. * (double)data_err[r + 1] * data_err[r + 1] * mock[r + 1] * cimag(t3der);
        }
        grad[q] = g;
    }
    free(ex);
    free(ey);
}

/* FP64 visibilities at selected uv points (same sum as o64_image2vis). */
void o64_image2vis_subset(int N, const double *image, const float *uv, float pix, int nsel, const int *sel,
                          double *visi)
{
    double F = 0;
    for (int i = 0; i < N * N; i++) F += image[i];
    double complex *V = (double complex *)visi;
    double complex *ex = malloc(sizeof(double complex) * N), *ey = malloc(sizeof(double complex) * N);
    for (int q = 0; q < nsel; q++) {
        const int k = sel[q];
        for (int i = 0; i < N; i++) {
            double px = o64_phase(pix, uv[4 * k], i), py = o64_phase(pix, uv[4 * k + 1], i);
            ex[i] = cos(px) + I * sin(px);
            ey[i] = cos(py) - I * sin(py);
        }
        double complex acc = 0;
        for (int y = 0; y < N; y++) {
            double complex row = 0;
            for (int x = 0; x < N; x++) row += image[y * N + x] * ex[x];
            acc += row * ey[y];
        }
        V[q] = (F > 0.) ? acc / F : acc;
    }
    free(ex);
    free(ey);
}
