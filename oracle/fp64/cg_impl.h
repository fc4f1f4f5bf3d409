/*
 * cg_impl.h -- restatement of the reference's GPU-path nonlinear conjugate
 * gradient with strong-Wolfe line search, instantiated for one scalar type.
 *
 * TEST INFRASTRUCTURE ONLY (oracle). Included by oracle_fp64.c twice:
 *   REAL=double, CG(name)=o64_##name  -- the FP64 oracle's CG;
 *   REAL=float,  CG(name)=o32_##name  -- the float CG that drives the
 *                                        reference's own cpu.c functions
 *                                        (the timed CPU baseline).
 *
 * Control flow follows, line by line in meaning:
 *   main CG loop        gpair1/trunk/gpair.c:682-915
 *   beta rules          gpair1/trunk/gpair.c:727-758 (0 SD, 1 FR, 2 PR+, 3 HS+,
 *                       restart when |g_new.g_old|/|g_new|^2 > 0.5)
 *   bracketing phase    gpair1/trunk/gpair.c:797-906
 *   zoom                gpair1/trunk/gpu.c:1947-2065 (quadratic step with
 *                       bisection fallback; J_lo is not updated inside zoom;
 *                       acceptance when wolfe2 >= c2*wolfe1 or counter > 10)
 *   image update        gpair1/trunk/gpair.c:910 (clamp at minvalue), then an
 *                       unconditional gradient backup (gpair1/trunk/gpair.c:913)
 * One deliberate difference: the zoom loop is capped at `max_zoom` trials.
 * The reference loop has no cap and can spin forever once hi and lo are
 * adjacent floating-point numbers; the cap only acts in that case.
 */

typedef struct {
    void *ctx;
    /* criterion J = chi2 - alpha*S of `image`; also returns chi2 and S */
    REAL (*criterion)(void *ctx, const REAL *image, REAL *chi2, REAL *entropy);
    /* full criterion gradient of `image` into `grad`; called only right after
     * criterion() on the same image, as the reference requires */
    void (*gradient)(void *ctx, const REAL *image, REAL *grad);
} CG(evaluator);

typedef struct {
    int method;        /* 0 SD, 1 FR, 2 PR+, 3 HS+; 4 projected L-BFGS (no reference counterpart) */
    int iterations;
    REAL minvalue;     /* 1e-8 */
    REAL wolfe1;       /* c1 = 1e-4 */
    REAL wolfe2;       /* c2 = 0.1 */
    REAL step_max;     /* 100 */
    int max_zoom;
} CG(params);

typedef struct {
    int criterion_evals, grad_evals;
    /* per iteration (arrays of length iterations, may be NULL) */
    REAL *J, *chi2, *entropy, *step, *beta;
} CG(trace);

static REAL CG(dot)(int n, const REAL *a, const REAL *b)
{
    REAL t = 0;
    for (int i = 0; i < n; i++) t += a[i] * b[i];
    return t;
}

static void CG(trial)(int n, const REAL *img, const REAL *d, REAL s, REAL minv, REAL *out)
{
    for (int i = 0; i < n; i++) {
        REAL t = img[i] + s * d[i];
        if (t < minv) t = minv;
        out[i] = t;
    }
}

static REAL CG(zoom)(const CG(evaluator) *ev, const CG(params) *p, int n, const REAL *img, const REAL *d,
                      REAL lo, REAL hi, REAL J_lo, REAL wolfe_product1, REAL J_init,
                      REAL *temp, REAL *tgrad, CG(trace) *tr)
{
    REAL s = 0, sel = 0, J = 0, J_old = 0, s_old = 0, chi2, S;
    int counter = 0;
    for (int guard = 0; guard < p->max_zoom; guard++) {
        if (counter > 0 && (J_old - J_init - wolfe_product1 * s_old) != 0)
            s = (REAL)fabs(wolfe_product1 * s_old * s_old / (2. * (J_old - J_init - wolfe_product1 * s_old)));
        if (counter == 0 || s < lo || s > hi)
            s = (hi - lo) / 2. + lo;
        if (fabs(hi - lo) < 1e-14) return lo;
        CG(trial)(n, img, d, s, p->minvalue, temp);
        J = ev->criterion(ev->ctx, temp, &chi2, &S);
        tr->criterion_evals++;
        if ((J > (J_init + p->wolfe1 * s * wolfe_product1)) || (J >= J_lo)) {
            hi = s;
        } else {
            ev->gradient(ev->ctx, temp, tgrad);
            tr->grad_evals++;
            REAL wolfe_product2 = CG(dot)(n, d, tgrad);
            if ((wolfe_product2 >= p->wolfe2 * wolfe_product1) || (counter > 10)) {
                sel = s;
                return sel;
            }
            if (wolfe_product2 * (hi - lo) >= 0.) hi = lo;
            lo = s;
        }
        s_old = s;
        J_old = J;
        counter++;
    }
    return lo;
}

/*
 * Batched line search (the library's GPAIR_LS_BATCH extension; the reference
 * has no counterpart). Same CG loop and beta rules as CG(run); each line
 * search evaluates rounds of LSB_NTR trial steps:
 *   grid round    s_c * 4^(j-3), j = 0..7 (s_c: the last accepted step, 1 at start)
 *   no decrease   move the grid below the smallest step tried (s_c / 4^5 of it)
 *   best = top    move the grid above the best step (s_c = best * 4^4)
 *   bracketed     one refine round of 8 evenly spaced steps inside (lo, hi),
 *                 the evaluated neighbours of the best step
 *   accept        the best step over all rounds (ties: the smaller step)
 * at most LSB_ROUNDS rounds; a direction that is not a descent direction, or
 * a search without any decrease, takes no step and restarts from -g.
 */
#ifndef LSB_NTR
#define LSB_NTR 8
#define LSB_ROUNDS 6
#define LSB_RATIO 4.0
#endif

static REAL CG(batch_search)(const CG(evaluator) *ev, const CG(params) *p, int n, const REAL *img, const REAL *d,
                             REAL J_init, double *s_c, double step_cap, int *force_sd, REAL *temp, CG(trace) *tr)
{
    double ts[LSB_NTR], ps[LSB_NTR * LSB_ROUNDS], pJ[LSB_NTR * LSB_ROUNDS];
    int npts = 0, round = 0, refine = 0;
    for (int j = 0; j < LSB_NTR; j++) {
        double t = *s_c * pow(LSB_RATIO, (double)(j - 3));
        ts[j] = t < step_cap ? t : step_cap;
    }
    for (;;) {
        for (int j = 0; j < LSB_NTR; j++) {
            REAL chi2, S;
            CG(trial)(n, img, d, (REAL)ts[j], p->minvalue, temp);
            double J = ev->criterion(ev->ctx, temp, &chi2, &S);
            if (!isfinite(J)) J = INFINITY;
            ps[npts] = ts[j];
            pJ[npts] = J;
            npts++;
        }
        tr->criterion_evals += LSB_NTR;
        round++;
        int b = -1;
        double sb = 0.0, Jb = J_init;
        for (int i = 0; i < npts; i++)
            if (pJ[i] < Jb || (pJ[i] == Jb && b >= 0 && ps[i] < sb)) { b = i; sb = ps[i]; Jb = pJ[i]; }
        if (b < 0) {
            double smin = ps[0];
            for (int i = 1; i < npts; i++) smin = fmin(smin, ps[i]);
            if (round < LSB_ROUNDS && smin > 1e-300) {
                *s_c = smin / pow(LSB_RATIO, 5.0);
                for (int j = 0; j < LSB_NTR; j++) {
                    double t = *s_c * pow(LSB_RATIO, (double)(j - 3));
                    ts[j] = t < step_cap ? t : step_cap;
                }
                continue;
            }
            *force_sd = 1;
            return 0;
        }
        double lo = 0.0, hi = INFINITY;
        for (int i = 0; i < npts; i++) {
            if (ps[i] < sb && ps[i] > lo) lo = ps[i];
            if (ps[i] > sb && ps[i] < hi) hi = ps[i];
        }
        if (!(hi < INFINITY)) {
            if (round < LSB_ROUNDS - 1 && sb < step_cap) {
                *s_c = sb * pow(LSB_RATIO, 4.0);
                for (int j = 0; j < LSB_NTR; j++) {
                    double t = *s_c * pow(LSB_RATIO, (double)(j - 3));
                    ts[j] = t < step_cap ? t : step_cap;
                }
                continue;
            }
        } else if (!refine && round < LSB_ROUNDS) {
            refine = 1;
            for (int j = 0; j < LSB_NTR; j++) ts[j] = lo + (hi - lo) * (double)(j + 1) / (double)(LSB_NTR + 1);
            continue;
        }
        if (sb > 0.0) *s_c = sb;
        return (REAL)sb;
    }
}

/*
 * Projected limited-memory BFGS direction (batched search, method 4; no
 * counterpart in the reference or the library yet). Pixels on the positivity
 * bound whose gradient points outward are held fixed: the gradient is zeroed
 * there before the two-loop recursion (Nocedal & Wright, Algorithm 7.4) and
 * the direction after it. The pairs s = x_new - x_old (the step actually
 * taken, after the clamp) and y = g_new - g_old are kept when s.y > 1e-12 |s| |y|;
 * H0 = (s.y / y.y) I from the newest pair.
 */
#define LBFGS_PAIRS 4

typedef struct {
    REAL *s, *y, *x_old;   /* LBFGS_PAIRS * n each for s and y; n for x_old */
    double rho[LBFGS_PAIRS], gamma;
    int head, count;       /* pairs stored: count <= LBFGS_PAIRS, newest at (head - 1) */
} CG(lbfgs);

static int CG(lbfgs_init)(CG(lbfgs) *L, int n)
{
    memset(L, 0, sizeof(*L));
    L->gamma = 1.0;
    L->s = calloc((size_t)LBFGS_PAIRS * n, sizeof(REAL));
    L->y = calloc((size_t)LBFGS_PAIRS * n, sizeof(REAL));
    L->x_old = calloc((size_t)n, sizeof(REAL));
    return (L->s && L->y && L->x_old) ? 0 : -1;
}

static void CG(lbfgs_free)(CG(lbfgs) *L) { free(L->s); free(L->y); free(L->x_old); }

/* new pair from the last step (x_old -> image, g_old -> g_new); a rejected pair
 * leaves every stored pair untouched (the candidate is formed in place only
 * once it is accepted) */
static void CG(lbfgs_update)(CG(lbfgs) *L, int n, const REAL *image, const REAL *g_new, const REAL *g_old)
{
    REAL sy = 0, yy = 0, ss = 0;
    for (int i = 0; i < n; i++) {
        const REAL si = image[i] - L->x_old[i], yi = g_new[i] - g_old[i];
        sy += si * yi;
        yy += yi * yi;
        ss += si * si;
    }
    if (yy > 0 && sy > 1e-12 * sqrt(ss * yy)) {
        REAL *sk = L->s + (size_t)(L->head % LBFGS_PAIRS) * n, *yk = L->y + (size_t)(L->head % LBFGS_PAIRS) * n;
        for (int i = 0; i < n; i++) { sk[i] = image[i] - L->x_old[i]; yk[i] = g_new[i] - g_old[i]; }
        L->rho[L->head % LBFGS_PAIRS] = 1.0 / sy;
        L->gamma = sy / yy;
        L->head++;
        if (L->count < LBFGS_PAIRS) L->count++;
    }
}

static void CG(lbfgs_dir)(const CG(lbfgs) *L, int n, const REAL *image, const REAL *g, REAL minvalue, REAL *d)
{
    double al[LBFGS_PAIRS];
    const REAL bound = minvalue * (REAL)1.000001;
    for (int i = 0; i < n; i++) d[i] = (image[i] <= bound && g[i] > 0) ? 0 : g[i];
    for (int j = 0; j < L->count; j++) {
        const int slot = (L->head - 1 - j) % LBFGS_PAIRS;
        const REAL *sk = L->s + (size_t)slot * n, *yk = L->y + (size_t)slot * n;
        al[j] = L->rho[slot] * CG(dot)(n, sk, d);
        for (int i = 0; i < n; i++) d[i] -= (REAL)al[j] * yk[i];
    }
    if (L->count)
        for (int i = 0; i < n; i++) d[i] *= (REAL)L->gamma;
    for (int j = L->count - 1; j >= 0; j--) {
        const int slot = (L->head - 1 - j) % LBFGS_PAIRS;
        const REAL *sk = L->s + (size_t)slot * n, *yk = L->y + (size_t)slot * n;
        const double b = L->rho[slot] * CG(dot)(n, yk, d);
        for (int i = 0; i < n; i++) d[i] += (REAL)(al[j] - b) * sk[i];
    }
    for (int i = 0; i < n; i++) d[i] = (image[i] <= bound && g[i] > 0) ? 0 : -d[i];
}

static int CG(run_batch)(const CG(evaluator) *ev, const CG(params) *p, int n, REAL *image, CG(trace) *tr,
                         double step_cap)
{
    REAL *g_new = calloc(n, sizeof(REAL)), *g_old = calloc(n, sizeof(REAL));
    REAL *d = calloc(n, sizeof(REAL)), *temp = calloc(n, sizeof(REAL));
    if (!g_new || !g_old || !d || !temp) return -1;
    REAL beta = 0, chi2, S;
    double s_c = 1.0;
    int force_sd = 0;
    const int lbfgs = p->method == 4;
    CG(lbfgs) L;
    if (lbfgs && CG(lbfgs_init)(&L, n)) return -1;
    tr->criterion_evals = tr->grad_evals = 0;
    for (int it = 0; it < p->iterations; it++) {
        REAL J = ev->criterion(ev->ctx, image, &chi2, &S);
        tr->criterion_evals++;
        ev->gradient(ev->ctx, image, g_new);
        tr->grad_evals++;
        if (it == 0 || p->method == 0 || lbfgs) {
            beta = 0.;
        } else {
            REAL nn = CG(dot)(n, g_new, g_new), no = CG(dot)(n, g_new, g_old), oo = CG(dot)(n, g_old, g_old);
            if (p->method == 1) beta = nn / oo;
            if (p->method == 2) { beta = (nn - no) / oo; if (beta < 0.) beta = 0.; }
            if (p->method == 3) {
                beta = (nn - no) / (CG(dot)(n, d, g_new) - CG(dot)(n, d, g_old));
                if (beta < 0.) beta = 0.;
            }
            if (fabs(no / nn) > .5) beta = 0.;
        }
        if (lbfgs) {
            if (it > 0) CG(lbfgs_update)(&L, n, image, g_new, g_old);
            if (force_sd) { L.count = 0; force_sd = 0; }  /* a failed search drops the history */
            CG(lbfgs_dir)(&L, n, image, g_new, p->minvalue, d);
        } else {
            if (force_sd) { beta = 0.; force_sd = 0; }
            for (int i = 0; i < n; i++) d[i] = beta * d[i] - g_new[i];
        }
        if (tr->J) { tr->J[it] = J; tr->chi2[it] = chi2; tr->entropy[it] = S; tr->beta[it] = beta; }
        REAL w1 = CG(dot)(n, d, g_new), sel = 0;
        if (!(w1 < 0)) {
            force_sd = 1;
        } else {
            /* A quasi-Newton direction carries its own scale: centre the grid on
             * step 1. Centred on the last CG-scale step instead, the trial images
             * of a float evaluation round back to the current image, show no
             * decrease, and the search moves the grid further down and fails. */
            if (lbfgs && L.count > 0) s_c = 1.0;
            sel = CG(batch_search)(ev, p, n, image, d, J, &s_c, step_cap, &force_sd, temp, tr);
        }
        if (tr->step) tr->step[it] = sel;
        if (lbfgs) memcpy(L.x_old, image, sizeof(REAL) * n);
        CG(trial)(n, image, d, sel, p->minvalue, image);
        memcpy(g_old, g_new, sizeof(REAL) * n);
    }
    if (lbfgs) CG(lbfgs_free)(&L);
    free(g_new); free(g_old); free(d); free(temp);
    return 0;
}

/* Runs p->iterations CG iterations on `image` (updated in place). */
static int CG(run)(const CG(evaluator) *ev, const CG(params) *p, int n, REAL *image, CG(trace) *tr)
{
    REAL *g_new = calloc(n, sizeof(REAL)), *g_old = calloc(n, sizeof(REAL));
    REAL *d = calloc(n, sizeof(REAL)), *temp = calloc(n, sizeof(REAL)), *tgrad = calloc(n, sizeof(REAL));
    if (!g_new || !g_old || !d || !temp || !tgrad) return -1;
    CG(lbfgs) L;
    if (p->method == 4 && CG(lbfgs_init)(&L, n)) return -1;
    REAL beta = 0, sel = 0, chi2, S;
    tr->criterion_evals = tr->grad_evals = 0;
    for (int it = 0; it < p->iterations; it++) {
        REAL J = ev->criterion(ev->ctx, image, &chi2, &S);
        tr->criterion_evals++;
        ev->gradient(ev->ctx, image, g_new);
        tr->grad_evals++;
        if (it == 0 || p->method == 0) {
            beta = 0.;
        } else {
            REAL nn = CG(dot)(n, g_new, g_new), no = CG(dot)(n, g_new, g_old), oo = CG(dot)(n, g_old, g_old);
            if (p->method == 1) beta = nn / oo;
            if (p->method == 2) { beta = (nn - no) / oo; if (beta < 0.) beta = 0.; }
            if (p->method == 3) {
                beta = (nn - no) / (CG(dot)(n, d, g_new) - CG(dot)(n, d, g_old));
                if (beta < 0.) beta = 0.;
            }
            if (fabs(no / nn) > .5) beta = 0.;
        }
        if (tr->J) { tr->J[it] = J; tr->chi2[it] = chi2; tr->entropy[it] = S; tr->beta[it] = beta; }
        if (p->method == 4) {
            /* projected L-BFGS with the reference's search; a direction that is
             * not a descent direction falls back to the projected -g */
            if (it > 0) CG(lbfgs_update)(&L, n, image, g_new, g_old);
            CG(lbfgs_dir)(&L, n, image, g_new, p->minvalue, d);
            if (!(CG(dot)(n, d, g_new) < 0)) {
                L.count = 0;
                CG(lbfgs_dir)(&L, n, image, g_new, p->minvalue, d);
            }
            memcpy(L.x_old, image, sizeof(REAL) * n);
        } else {
            for (int i = 0; i < n; i++) d[i] = beta * d[i] - g_new[i];
        }
        REAL wolfe_product1 = CG(dot)(n, d, g_new);
        REAL s = 1., s_old = 0., J_init = J, J_old = J, Jt;
        int ls_it = 1;
        sel = 0.;
        while (1) {
            CG(trial)(n, image, d, s, p->minvalue, temp);
            Jt = ev->criterion(ev->ctx, temp, &chi2, &S);
            tr->criterion_evals++;
            if ((Jt > (J_init + p->wolfe1 * s * wolfe_product1)) || ((Jt >= J_old) && (ls_it > 1))) {
                sel = CG(zoom)(ev, p, n, image, d, s_old, s, J_old, wolfe_product1, J_init, temp, tgrad, tr);
                break;
            }
            ev->gradient(ev->ctx, temp, tgrad);
            tr->grad_evals++;
            REAL wolfe_product2 = CG(dot)(n, d, tgrad);
            if (fabs(wolfe_product2) <= -p->wolfe2 * wolfe_product1) { sel = s; break; }
            if (wolfe_product2 >= 0.) {
                sel = CG(zoom)(ev, p, n, image, d, s, s_old, Jt, wolfe_product1, J_init, temp, tgrad, tr);
                break;
            }
            s_old = s;
            J_old = Jt;
            s = 10.0 * s;
            if (s > p->step_max) s = p->step_max;
            ls_it++;
        }
        if (tr->step) tr->step[it] = sel;
        CG(trial)(n, image, d, sel, p->minvalue, image);
        memcpy(g_old, g_new, sizeof(REAL) * n);
    }
    if (p->method == 4) CG(lbfgs_free)(&L);
    free(g_new); free(g_old); free(d); free(temp); free(tgrad);
    return 0;
}
