// context.cu -- device contexts, problem upload and the evaluation / CG
// orchestration behind the extension API of gpair_b200.h.
//
// One criterion evaluation (gpair_criterion) = k_prep -> forward DFT ->
// k_vis_data; one gradient evaluation (gpair_gradient) = k_adj_weights ->
// adjoint DFT -> k_grad_finalize. gpair_cg_run chains them with the device
// controller k_cg_ctrl, which holds every CG scalar in FP64 on the GPU; the
// host only reads back the controller's next action (evaluate criterion,
// evaluate gradient, or accept the step).
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "gpair_internal.cuh"

int gp_default_splits(int N, int nuv);
void gp_cg_graph_free(gpair_ctx *c);
int gp_cg_graph_run(gpair_ctx *c, int iterations, int want_trace, int ls_mode, long long *launches);
int gp_cg_graph_trace(gpair_ctx *c, int iterations, double *tJ, double *tchi2, double *tS, double *tstep,
                      double *tbeta);
long long gp_cg_graph_launches(gpair_ctx *c, int iterations_done, int criterion_evals, int grad_evals, int batches);
int gp_batch_graph_build(gpair_ctx **ctx, int n, int ls_mode, int allow_group, void **out);
void gp_batch_graph_free(void *bg);
int gp_batch_graph_launch(void *bg, cudaStream_t stream);
int gp_batch_graph_precision(void *bg, int i);
unsigned int gp_batch_graph_buf_gen(void *bg, int i);
int gp_batch_graph_grouped(void *bg);
int gp_batch_graph_prep_passes(void *bg);
int gp_batch_graph_stamps(void *bg, unsigned long long *out, int max, cudaStream_t st, int reset);
long long gp_batch_graph_launches(void *bg, int i, int iterations_done, int criterion_evals, int grad_evals,
                                  int batches);

static const char *k_err_names[] = {"GPAIR_OK",      "GPAIR_ERR_INVALID", "GPAIR_ERR_ALLOC",     "GPAIR_ERR_CUDA",
                                    "GPAIR_ERR_STATE", "GPAIR_ERR_TIMEOUT", "GPAIR_ERR_NO_DEVICE", "GPAIR_ERR_NUMERIC"};

extern "C" const char *gpair_strerror(int status)
{
    int i = -status;
    if (i < 0 || i >= (int)(sizeof(k_err_names) / sizeof(k_err_names[0]))) return "GPAIR_ERR_UNKNOWN";
    return k_err_names[i];
}

extern "C" const char *gpair_last_error(gpair_ctx *ctx) { return ctx ? ctx->last_error : "no context"; }

#define FREE_DEV(p)              \
    do {                         \
        if (p) cudaFree(p);      \
        (p) = nullptr;           \
    } while (0)

static void free_problem(gpair_ctx *c)
{
    gp_cg_graph_free(c);
    FREE_DEV(c->data); FREE_DEV(c->data_err); FREE_DEV(c->mock);
    FREE_DEV(c->tri); FREE_DEV(c->phasor); FREE_DEV(c->uvc);
    FREE_DEV(c->fx); FREE_DEV(c->fy); FREE_DEV(c->vpart); FREE_DEV(c->visd); FREE_DEV(c->visi);
    FREE_DEV(c->trib); FREE_DEV(c->cw); FREE_DEV(c->inc_off); FREE_DEV(c->inc_idx); FREE_DEV(c->gpart);
    gp_batch_free(c);
    gp_tc_free(c);
    c->have_problem = 0;
}

static void free_images(gpair_ctx *c)
{
    gp_cg_graph_free(c);
    FREE_DEV(c->image); FREE_DEV(c->image_temp); FREE_DEV(c->model);
    FREE_DEV(c->data_grad); FREE_DEV(c->entropy_grad); FREE_DEV(c->full_grad_new);
    FREE_DEV(c->full_grad); FREE_DEV(c->grad_temp); FREE_DEV(c->descent_dir);
    gp_batch_free(c);
    gp_lbfgs_free(c);
    c->N = 0;
    c->npix = 0;
    c->have_image = 0;
}

static void set_handle(gpair_buf *h, float *p, size_t n, int id)
{
    h->ptr = p;
    h->count = n;
    h->id = id;
}

// (Re)allocate the image-sized buffers for width N; contents are zeroed.
int gp_alloc_images(gpair_ctx *c, int N)
{
    if (N <= 0 || (long long)N * N > (1LL << 30)) return GPAIR_ERR_INVALID;
    if (c->N == N && c->image) return GPAIR_OK;
    GP_CUDA(c, cudaSetDevice(c->device));
    free_images(c);
    size_t n = (size_t)N * N, bytes = n * sizeof(float);
    float **bufs[] = {&c->image, &c->image_temp, &c->model, &c->data_grad, &c->entropy_grad,
                      &c->full_grad_new, &c->full_grad, &c->grad_temp, &c->descent_dir};
    for (float **b : bufs) {
        GP_CUDA(c, cudaMalloc(b, bytes));
        GP_CUDA(c, cudaMemsetAsync(*b, 0, bytes, c->stream));
    }
    c->N = N;
    c->npix = (int)n;
    set_handle(&c->h_image, c->image, n, 0);
    set_handle(&c->h_image_temp, c->image_temp, n, 1);
    set_handle(&c->h_fgn, c->full_grad_new, n, 2);
    set_handle(&c->h_fg, c->full_grad, n, 3);
    set_handle(&c->h_dd, c->descent_dir, n, 4);
    set_handle(&c->h_tg, c->grad_temp, n, 5);
    set_handle(&c->h_eg, c->entropy_grad, n, 6);
    set_handle(&c->h_dg, c->data_grad, n, 7);
    set_handle(&c->h_model, c->model, n, 8);
    return GPAIR_OK;
}

extern "C" int gpair_create(gpair_ctx **out, int device)
{
    if (!out) return GPAIR_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return GPAIR_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return GPAIR_ERR_NO_DEVICE;
    if (prop.major != 10) return GPAIR_ERR_NO_DEVICE;  // built for sm_100a only
    gpair_ctx *c = (gpair_ctx *)calloc(1, sizeof(gpair_ctx));
    if (!c) return GPAIR_ERR_ALLOC;
    c->device = device;
    c->precision = GPAIR_PREC_FP32;
    c->tc_pair = 1;  // tensor-core contractions on CTA pairs (gpair_set_tc_pair)
    c->gf_parts = 8;
    {
        const char *e = getenv("GPAIR_PDL");  // programmatic dependent launches (gpair_set_pdl)
        c->pdl = (e && e[0] == '0') ? 0 : 1;
    }
    c->fuse_ctrl = -1;
    c->last_image_src = -1;
    int rc = GPAIR_OK;
    do {
        if (cudaSetDevice(device) != cudaSuccess) { rc = GPAIR_ERR_CUDA; break; }
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { rc = GPAIR_ERR_CUDA; break; }
        if (cudaMalloc(&c->sc, sizeof(DevScalars)) != cudaSuccess) { rc = GPAIR_ERR_ALLOC; break; }
        if (cudaMemset(c->sc, 0, sizeof(DevScalars)) != cudaSuccess) { rc = GPAIR_ERR_CUDA; break; }
        if (cudaMallocHost(&c->sc_host, sizeof(DevScalars)) != cudaSuccess) { rc = GPAIR_ERR_ALLOC; break; }
        size_t pbytes = sizeof(double) * RED_NSLOTS * GP_MAX_PARTIALS * 4;
        if (cudaMalloc(&c->partials, pbytes) != cudaSuccess) { rc = GPAIR_ERR_ALLOC; break; }
    } while (0);
    if (rc != GPAIR_OK) {
        gpair_destroy(c);
        return rc;
    }
    *out = c;
    return GPAIR_OK;
}

extern "C" int gpair_destroy(gpair_ctx *c)
{
    if (!c) return GPAIR_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_problem(c);
    free_images(c);
    FREE_DEV(c->sc);
    FREE_DEV(c->partials);
    if (c->sc_host) cudaFreeHost(c->sc_host);
    if (c->st_ev) {
        for (int i = 0; i < 2 * GP_MAX_STAGE_REC; i++)
            if (c->st_ev[i]) cudaEventDestroy(c->st_ev[i]);
        free(c->st_ev);
        free(c->st_stage);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    free(c->ref_dft_x); free(c->ref_dft_y); free(c->ref_data); free(c->ref_data_err); free(c->ref_model);
    free(c->ref_phasor); free(c->ref_uvpnt); free(c->ref_sign);
    free(c);
    return GPAIR_OK;
}

// CSR map uv point -> incident (triangle, vertex) slots, ascending (t, vertex)
int gp_build_incidence(gpair_ctx *c, const int64_t *uvpnt)
{
    std::vector<int> off(c->nuv + 1, 0), idx((size_t)3 * c->nbis);
    for (long long j = 0; j < 3LL * c->nbis; j++) off[uvpnt[j] + 1]++;
    for (int k = 0; k < c->nuv; k++) off[k + 1] += off[k];
    std::vector<int> pos(off.begin(), off.end() - 1);
    for (long long j = 0; j < 3LL * c->nbis; j++) idx[pos[uvpnt[j]]++] = (int)j;
    GP_CUDA(c, cudaMalloc(&c->inc_off, sizeof(int) * (c->nuv + 1)));
    GP_CUDA(c, cudaMalloc(&c->inc_idx, sizeof(int) * (idx.empty() ? 1 : idx.size())));
    GP_CUDA(c, cudaMemcpyAsync(c->inc_off, off.data(), sizeof(int) * (c->nuv + 1), cudaMemcpyHostToDevice, c->stream));
    if (!idx.empty())
        GP_CUDA(c, cudaMemcpyAsync(c->inc_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

// Problem upload. uv may be NULL when the twiddles are supplied as tables
// afterwards (reference boundary path, gpu_copy_dft).
int gp_set_problem_core(gpair_ctx *c, int N, float pix, int nuv, const gpair_uv *uv, int npow, int nbis,
                        const float *data, const float *data_err, const gpair_float2 *phasor, const int64_t *uvpnt,
                        const int16_t *sign, const float *model)
{
    if (!c || N <= 0 || nuv < 0 || npow < 0 || nbis < 0 || npow > nuv) return GPAIR_ERR_INVALID;
    if ((npow + 2LL * nbis) > (1LL << 31) - 1 || (long long)nuv * N > (1LL << 31)) return GPAIR_ERR_INVALID;
    if ((npow + nbis) > 0 && (!data || !data_err)) return GPAIR_ERR_INVALID;
    if (nbis > 0 && (!phasor || !uvpnt || !sign)) return GPAIR_ERR_INVALID;
    for (long long j = 0; j < 3LL * nbis; j++)
        if (uvpnt[j] < 0 || uvpnt[j] >= nuv) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    int rc = gp_alloc_images(c, N);
    if (rc) return rc;
    free_problem(c);
    GP_CUDA(c, cudaMemsetAsync(&c->sc->nonfinite, 0, sizeof(unsigned int), c->stream));
    c->pix = pix;
    c->nuv = nuv;
    c->npow = npow;
    c->nbis = nbis;
    c->ndata = npow + 2 * nbis;
    size_t nd = c->ndata ? c->ndata : 1, nt = nbis ? nbis : 1, nk = nuv ? nuv : 1;
    c->mt = gp_cdiv(N, 64);
    c->splits_simt = gp_default_splits(N, nuv ? nuv : 1);
    c->splits = c->splits_simt;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    int max_splits = gp_tc_max_splits(N, nuv ? nuv : 1, nsm);
    if (max_splits < c->splits_simt) max_splits = c->splits_simt;
    GP_CUDA(c, cudaMalloc(&c->data, nd * sizeof(float)));
    GP_CUDA(c, cudaMalloc(&c->data_err, nd * sizeof(float)));
    GP_CUDA(c, cudaMalloc(&c->mock, nd * sizeof(float)));
    GP_CUDA(c, cudaMalloc(&c->tri, nt * sizeof(int4)));
    GP_CUDA(c, cudaMalloc(&c->phasor, nt * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->uvc, nk * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->fx, nk * N * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->fy, nk * N * sizeof(float2)));
    // partial visibility entries: the CUDA-core forward's row tiles or the tensor forward's entries
    const int mt_cap = c->mt > gp_tc_forward_entries(N) ? c->mt : gp_tc_forward_entries(N);
    GP_CUDA(c, cudaMalloc(&c->vpart, (size_t)mt_cap * nk * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->visd, nk * sizeof(double2)));
    GP_CUDA(c, cudaMalloc(&c->visi, nk * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->cw, nk * sizeof(float2)));
    GP_CUDA(c, cudaMalloc(&c->trib, 3 * nt * sizeof(float2)));
    // room for twice the default split count: the autotuner may shorten the split-K tiles
    c->gpart_cap = 2 * max_splits;
    GP_CUDA(c, cudaMalloc(&c->gpart, (size_t)c->gpart_cap * c->npix * sizeof(float)));
    GP_CUDA(c, cudaMemsetAsync(c->mock, 0, nd * sizeof(float), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->visd, 0, nk * sizeof(double2), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->visi, 0, nk * sizeof(float2), c->stream));
    if (c->ndata) {
        GP_CUDA(c, cudaMemcpyAsync(c->data, data, c->ndata * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        GP_CUDA(c, cudaMemcpyAsync(c->data_err, data_err, c->ndata * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    }
    std::vector<int4> tri(nt);
    for (int t = 0; t < nbis; t++) {
        int w = (sign[3 * t] < 0 ? 1 : 0) | (sign[3 * t + 1] < 0 ? 2 : 0) | (sign[3 * t + 2] < 0 ? 4 : 0);
        tri[t] = make_int4((int)uvpnt[3 * t], (int)uvpnt[3 * t + 1], (int)uvpnt[3 * t + 2], w);
    }
    if (nbis) {
        GP_CUDA(c, cudaMemcpyAsync(c->tri, tri.data(), nbis * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
        GP_CUDA(c, cudaMemcpyAsync(c->phasor, phasor, nbis * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    }
    if (model)
        GP_CUDA(c, cudaMemcpyAsync(c->model, model, c->npix * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    // the entropy-gradient buffer starts at zero: where image <= 0 or model <= 0
    // it keeps its previous value (gpair1/trunk/gpu.c:1332-1338, kernel_entropy_gs_grad.cl)
    GP_CUDA(c, cudaMemsetAsync(c->entropy_grad, 0, c->npix * sizeof(float), c->stream));
    // a new problem starts without CG history (same-width image buffers are reused)
    GP_CUDA(c, cudaMemsetAsync(c->descent_dir, 0, c->npix * sizeof(float), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->full_grad, 0, c->npix * sizeof(float), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->full_grad_new, 0, c->npix * sizeof(float), c->stream));
    c->have_uv = uv && nuv;
    if (uv && nuv) {
        std::vector<float2> uvc(nuv);
        for (int k = 0; k < nuv; k++) uvc[k] = make_float2(uv[k].u, uv[k].v);
        GP_CUDA(c, cudaMemcpyAsync(c->uvc, uvc.data(), nuv * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
        rc = gp_gen_twiddles(c);
        if (rc) return rc;
    }
    rc = gp_build_incidence(c, uvpnt);
    if (rc) return rc;
    c->have_problem = 1;
    if (c->precision != GPAIR_PREC_FP32 && uv) {
        // with reference tables (uv == NULL) the operands are built lazily, once the tables are on the device
        rc = gp_tc_prepare(c);
        if (rc) return rc;
    }
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

extern "C" int gpair_set_problem(gpair_ctx *c, int N, float pix, int nuv, const gpair_uv *uv, int npow, int nbis,
                                 const float *data, const float *data_err, const gpair_float2 *phasor,
                                 const int64_t *uvpnt, const int16_t *sign, const float *model)
{
    if (!uv && nuv > 0) return GPAIR_ERR_INVALID;
    return gp_set_problem_core(c, N, pix, nuv, uv, npow, nbis, data, data_err, phasor, uvpnt, sign, model);
}

extern "C" int gpair_set_precision(gpair_ctx *c, int mode)
{
    if (!c || mode < GPAIR_PREC_FP32 || mode > GPAIR_PREC_SPLIT16F8) return GPAIR_ERR_INVALID;
    int old = c->precision;
    c->precision = mode;
    if (mode != GPAIR_PREC_FP32 && c->have_problem) {
        int rc = gp_tc_prepare(c);
        if (rc) {
            c->precision = old;
            return rc;
        }
    }
    return GPAIR_OK;
}

extern "C" int gpair_get_precision(gpair_ctx *c) { return c ? c->precision : -1; }

extern "C" int gpair_set_image(gpair_ctx *c, int which, const float *image)
{
    if (!c || !image || !c->image) return GPAIR_ERR_STATE;
    float *dst = which == GPAIR_IMG_TEMP ? c->image_temp : c->image;
    GP_CUDA(c, cudaMemcpyAsync(dst, image, c->npix * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_image = 1;
    return GPAIR_OK;
}

static int d2h(gpair_ctx *c, void *dst, const void *src, size_t bytes)
{
    GP_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

extern "C" int gpair_get_image(gpair_ctx *c, int which, float *image)
{
    if (!c || !image || !c->image) return GPAIR_ERR_STATE;
    return d2h(c, image, which == GPAIR_IMG_TEMP ? c->image_temp : c->image, c->npix * sizeof(float));
}

int gp_sync_scalars(gpair_ctx *c)
{
    GP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->sc_host->tc_err) {
        // a tensor-core kernel gave up a bounded wait; report it once and clear it
        snprintf(c->last_error, sizeof(c->last_error), "tensor-core kernel wait timed out (code 0x%x)",
                 c->sc_host->tc_err);
        unsigned int zero = 0;
        cudaMemcpyAsync(&c->sc->tc_err, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
        return GPAIR_ERR_TIMEOUT;
    }
    return GPAIR_OK;
}

// ----------------------------------------------------------- stage timing

void gp_stage_begin(gpair_ctx *c, int stage)
{
    if (!c->stage_timing || !c->st_ev || c->st_n >= GP_MAX_STAGE_REC) return;
    c->st_stage[c->st_n] = stage;
    cudaEventRecord(c->st_ev[2 * c->st_n], c->stream);
}

void gp_stage_end(gpair_ctx *c)
{
    if (!c->stage_timing || !c->st_ev || c->st_n >= GP_MAX_STAGE_REC) return;
    cudaEventRecord(c->st_ev[2 * c->st_n + 1], c->stream);
    c->st_n++;
}

static void stage_collect(gpair_ctx *c)
{
    for (int i = 0; i < 8; i++) { c->stage_ms[i] = 0.0; c->stage_cnt[i] = 0; }
    for (int r = 0; r < c->st_n; r++) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, c->st_ev[2 * r], c->st_ev[2 * r + 1]) == cudaSuccess) {
            c->stage_ms[c->st_stage[r]] += t;
            c->stage_cnt[c->st_stage[r]]++;
        }
    }
    c->st_n = 0;
}

extern "C" int gpair_set_tc_pair(gpair_ctx *c, int on)
{
    if (!c) return GPAIR_ERR_INVALID;
    c->tc_pair = on ? 1 : 0;
    gp_cg_graph_free(c);  // captured graphs hold the other kernel variant
    if (c->precision != GPAIR_PREC_FP32 && c->have_problem && c->have_uv) return gp_tc_prepare(c);
    return GPAIR_OK;
}

extern "C" int gpair_get_tc_pair(gpair_ctx *c) { return c ? c->tc_pair : -1; }

extern "C" int gpair_set_shared_splits(gpair_ctx **ctx, int n)
{
    if (!ctx || n < 1) return GPAIR_ERR_INVALID;
    for (int i = 0; i < n; i++)
        if (!ctx[i] || ctx[i]->device != ctx[0]->device) return GPAIR_ERR_INVALID;
    GP_CUDA(ctx[0], cudaSetDevice(ctx[0]->device));
    return gp_tc_shared_splits(ctx, n);
}

extern "C" int gpair_set_pdl(gpair_ctx *c, int on)
{
    if (!c) return GPAIR_ERR_INVALID;
    c->pdl = on ? 1 : 0;
    gp_cg_graph_free(c);  // captured graphs hold the launch attribute
    return GPAIR_OK;
}

extern "C" int gpair_set_tc_wait(gpair_ctx *c, long long budget_cycles, int skip_loads)
{
    if (!c || budget_cycles < 0) return GPAIR_ERR_INVALID;
    c->tc_wait_budget = budget_cycles;
    c->tc_skip_loads = skip_loads ? 1 : 0;
    return GPAIR_OK;
}

extern "C" int gpair_set_stage_timing(gpair_ctx *c, int on)
{
    if (!c) return GPAIR_ERR_INVALID;
    if (on && !c->st_ev) {
        GP_CUDA(c, cudaSetDevice(c->device));
        c->st_ev = (cudaEvent_t *)calloc(2 * GP_MAX_STAGE_REC, sizeof(cudaEvent_t));
        c->st_stage = (int *)calloc(GP_MAX_STAGE_REC, sizeof(int));
        if (!c->st_ev || !c->st_stage) return GPAIR_ERR_ALLOC;
        for (int i = 0; i < 2 * GP_MAX_STAGE_REC; i++) GP_CUDA(c, cudaEventCreate(&c->st_ev[i]));
    }
    c->stage_timing = on ? 1 : 0;
    c->st_n = 0;
    return GPAIR_OK;
}

extern "C" int gpair_last_run_stage_ms(gpair_ctx *c, double *ms, int *counts, int max_stages)
{
    if (!c || !ms) return GPAIR_ERR_INVALID;
    int n = max_stages < GPAIR_NSTAGES ? max_stages : GPAIR_NSTAGES;
    for (int i = 0; i < n; i++) {
        ms[i] = c->stage_ms[i];
        if (counts) counts[i] = c->stage_cnt[i];
    }
    return n;
}

// ----------------------------------------------------------- evaluations

int gp_eval_criterion(gpair_ctx *c, int which, int trial)
{
    int rc;
    gp_stage_begin(c, 0);
    // tensor path: image (or trial image), its sums and its forward operand in one pass
    const bool tc = c->precision != GPAIR_PREC_FP32;
    if (tc) rc = trial ? gp_tc_prep_split_trial(c) : gp_tc_prep_image(c, which);
    else rc = gp_prep_image(c, trial ? GPAIR_IMG_TEMP : which, trial, 0.0, trial);
    if (rc) return rc;
    gp_stage_end(c);
    gp_stage_begin(c, 1);
    if (tc) rc = gp_tc_forward_gemm(c);
    else rc = gp_forward(c, trial ? GPAIR_IMG_TEMP : which);
    if (rc) return rc;
    gp_stage_end(c);
    gp_stage_begin(c, 2);
    if ((rc = gp_vis_data(c))) return rc;
    gp_stage_end(c);
    c->last_image_src = trial ? GPAIR_IMG_TEMP : which;
    return GPAIR_OK;
}

int gp_eval_gradient(gpair_ctx *c, int which, float alpha)
{
    int rc;
    gp_stage_begin(c, 3);
    if ((rc = gp_adj_weights_only(c))) return rc;
    gp_stage_end(c);
    gp_stage_begin(c, 4);
    if ((rc = gp_adjoint_contraction(c, which))) return rc;
    gp_stage_end(c);
    gp_stage_begin(c, 5);
    rc = gp_grad_finalize(c, which, GRAD_FUSED, alpha);
    gp_stage_end(c);
    return rc;
}

extern "C" int gpair_criterion(gpair_ctx *c, int which, double *chi2, double *entropy)
{
    if (!c || !c->have_problem) return GPAIR_ERR_STATE;
    GP_CUDA(c, cudaSetDevice(c->device));
    // the non-finite flag describes this evaluation, not an earlier one
    GP_CUDA(c, cudaMemsetAsync(&c->sc->nonfinite, 0, sizeof(unsigned int), c->stream));
    int rc = gp_eval_criterion(c, which, 0);
    if (rc) return rc;
    if ((rc = gp_sync_scalars(c))) return rc;
    if (chi2) *chi2 = c->sc_host->chi2;
    if (entropy) *entropy = c->sc_host->entropy;
    return (c->sc_host->nonfinite & 3u) ? GPAIR_ERR_NUMERIC : GPAIR_OK;
}

extern "C" int gpair_gradient(gpair_ctx *c, int which, float alpha)
{
    if (!c || !c->have_problem || c->last_image_src < 0) return GPAIR_ERR_STATE;
    GP_CUDA(c, cudaSetDevice(c->device));
    int rc = gp_eval_gradient(c, which, alpha);
    if (rc) return rc;
    return gp_sync_scalars(c);
}

extern "C" int gpair_get_visibilities(gpair_ctx *c, gpair_float2 *visi)
{
    if (!c || !c->have_problem) return GPAIR_ERR_STATE;
    return d2h(c, visi, c->visi, sizeof(float2) * c->nuv);
}
extern "C" int gpair_get_mock(gpair_ctx *c, float *mock)
{
    if (!c || !c->have_problem) return GPAIR_ERR_STATE;
    return d2h(c, mock, c->mock, sizeof(float) * c->ndata);
}
extern "C" int gpair_get_data_gradient(gpair_ctx *c, float *g)
{
    if (!c || !c->image) return GPAIR_ERR_STATE;
    return d2h(c, g, c->data_grad, sizeof(float) * c->npix);
}
extern "C" int gpair_get_entropy_gradient(gpair_ctx *c, float *g)
{
    if (!c || !c->image) return GPAIR_ERR_STATE;
    return d2h(c, g, c->entropy_grad, sizeof(float) * c->npix);
}
extern "C" int gpair_get_full_gradient(gpair_ctx *c, int which, float *g)
{
    if (!c || !c->image) return GPAIR_ERR_STATE;
    return d2h(c, g, which == GPAIR_IMG_TEMP ? c->grad_temp : c->full_grad_new, sizeof(float) * c->npix);
}

// ---------------------------------------------------------------- CG

extern "C" void gpair_cg_default_params(gpair_cg_params *p)
{
    p->method = 2;
    p->iterations = 10;
    p->alpha = 1e-3f;
    p->minvalue = 1e-8;
    p->wolfe1 = 1e-4;
    p->wolfe2 = 0.1;
    p->step_max = 100.0;
    p->max_zoom = 200;
    p->max_bracket = 100;
    p->resume = 0;
    p->host_loop = 0;
    p->line_search = GPAIR_LS_WOLFE;
    p->target_J = 0.0;
    p->batch_step_max = 1e12;
    p->stop_flag = nullptr;
}

extern "C" int gpair_adjoint_image(gpair_ctx *c, const gpair_float2 *weights, float *image)
{
    if (!c || !c->have_problem || !weights || !image) return GPAIR_ERR_STATE;
    GP_CUDA(c, cudaSetDevice(c->device));
    c->last_image_src = -1;  // the evaluation state (weights, data gradient) is overwritten
    return gp_adjoint_image(c, (const float2 *)weights, image);
}

extern "C" int gpair_set_regularizer(gpair_ctx *c, int kind)
{
    if (!c || (kind != GPAIR_REG_GULL_SKILLING && kind != GPAIR_REG_L2)) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    GP_CUDA(c, cudaMemcpyAsync(&c->sc->reg_kind, &kind, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

extern "C" int gpair_update_pixel(gpair_ctx *c, int x, int y, float value, double *chi2, double *entropy)
{
    if (!c || !c->have_problem) return GPAIR_ERR_STATE;
    if (c->last_image_src != GPAIR_IMG_CURR) return GPAIR_ERR_STATE;  // V must be the current image's
    if (x < 0 || y < 0 || x >= c->N || y >= c->N || !(value == value)) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    GP_CUDA(c, cudaMemsetAsync(&c->sc->nonfinite, 0, sizeof(unsigned int), c->stream));
    int rc = gp_update_pixel(c, x, y, value);
    if (rc) return rc;
    if ((rc = gp_sync_scalars(c))) return rc;
    if (chi2) *chi2 = c->sc_host->chi2;
    if (entropy) *entropy = c->sc_host->entropy;
    return (c->sc_host->nonfinite & 3u) ? GPAIR_ERR_NUMERIC : GPAIR_OK;
}

// ---------------------------------------------------------- checkpoints
//
// Layout: CheckpointHeader, CgState (the device controller state), then float
// arrays of N*N: image, descent direction, previous gradient, current
// gradient, entropy gradient (kept where the regulariser keeps old values).
struct CheckpointHeader {
    char magic[8];  // "GPAIRCK1"
    int N, nuv, npow, nbis, precision, reg_kind;
    unsigned int cgstate_bytes, arrays;
};

static const int kCkArrays = 5;

extern "C" size_t gpair_cg_checkpoint_size(gpair_ctx *c)
{
    if (!c || !c->have_problem) return 0;
    return sizeof(CheckpointHeader) + sizeof(CgState) + (size_t)kCkArrays * c->npix * sizeof(float);
}

static float *ck_array(gpair_ctx *c, int i)
{
    float *a[kCkArrays] = {c->image, c->descent_dir, c->full_grad, c->full_grad_new, c->entropy_grad};
    return a[i];
}

extern "C" int gpair_cg_checkpoint_save(gpair_ctx *c, void *buf, size_t bytes)
{
    if (!c || !c->have_problem || !buf) return GPAIR_ERR_STATE;
    if (bytes < gpair_cg_checkpoint_size(c)) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    int rc = gp_sync_scalars(c);  // waits for the context's stream
    if (rc) return rc;
    CheckpointHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, "GPAIRCK1", 8);
    h.N = c->N;
    h.nuv = c->nuv;
    h.npow = c->npow;
    h.nbis = c->nbis;
    h.precision = c->precision;
    h.reg_kind = c->sc_host->reg_kind;
    h.cgstate_bytes = sizeof(CgState);
    h.arrays = kCkArrays;
    unsigned char *p = (unsigned char *)buf;
    memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    memcpy(p, &c->sc_host->cg, sizeof(CgState));
    p += sizeof(CgState);
    for (int i = 0; i < kCkArrays; i++) {
        GP_CUDA(c, cudaMemcpyAsync(p, ck_array(c, i), sizeof(float) * c->npix, cudaMemcpyDeviceToHost, c->stream));
        p += sizeof(float) * c->npix;
    }
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

extern "C" int gpair_cg_checkpoint_load(gpair_ctx *c, const void *buf, size_t bytes)
{
    if (!c || !c->have_problem || !buf) return GPAIR_ERR_STATE;
    if (bytes < gpair_cg_checkpoint_size(c)) return GPAIR_ERR_INVALID;
    CheckpointHeader h;
    memcpy(&h, buf, sizeof(h));
    if (memcmp(h.magic, "GPAIRCK1", 8) || h.cgstate_bytes != sizeof(CgState) || h.arrays != (unsigned)kCkArrays ||
        h.N != c->N || h.nuv != c->nuv || h.npow != c->npow || h.nbis != c->nbis) {
        snprintf(c->last_error, sizeof(c->last_error), "checkpoint does not match this problem or build");
        return GPAIR_ERR_INVALID;
    }
    GP_CUDA(c, cudaSetDevice(c->device));
    int rc = gpair_set_precision(c, h.precision);
    if (rc) return rc;
    if ((rc = gpair_set_regularizer(c, h.reg_kind))) return rc;
    const unsigned char *p = (const unsigned char *)buf + sizeof(h);
    // every copy on the context's stream, after the work already queued there;
    // the caller's buffer may be pageable, so wait until the last copy landed
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    // the projected L-BFGS pairs are not part of a checkpoint: a restored run
    // starts its history afresh (its first direction is the projected -g)
    memcpy(&c->sc_host->cg, p, sizeof(CgState));
    c->sc_host->cg.lb_count = 0;
    c->sc_host->cg.lb_xvalid = 0;
    c->sc_host->cg.lb_drop = 0;
    GP_CUDA(c, cudaMemcpyAsync(&c->sc->cg, &c->sc_host->cg, sizeof(CgState), cudaMemcpyHostToDevice, c->stream));
    p += sizeof(CgState);
    for (int i = 0; i < kCkArrays; i++) {
        GP_CUDA(c, cudaMemcpyAsync(ck_array(c, i), p, sizeof(float) * c->npix, cudaMemcpyHostToDevice, c->stream));
        p += sizeof(float) * c->npix;
    }
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->have_image = 1;
    c->last_image_src = -1;
    gp_cg_graph_free(c);
    return GPAIR_OK;
}

extern "C" int gpair_stop_flag_create(int **flag)
{
    if (!flag) return GPAIR_ERR_INVALID;
    if (cudaMalloc(flag, sizeof(int)) != cudaSuccess) return GPAIR_ERR_ALLOC;
    if (cudaMemset(*flag, 0, sizeof(int)) != cudaSuccess) return GPAIR_ERR_CUDA;
    return GPAIR_OK;
}

extern "C" int gpair_stop_flag_reset(int *flag)
{
    if (!flag) return GPAIR_ERR_INVALID;
    return cudaMemset(flag, 0, sizeof(int)) == cudaSuccess ? GPAIR_OK : GPAIR_ERR_CUDA;
}

extern "C" int gpair_stop_flag_destroy(int *flag)
{
    if (flag) cudaFree(flag);
    return GPAIR_OK;
}

static int read_action(gpair_ctx *c, int *action)
{
    GP_CUDA(c, cudaMemcpyAsync(&c->sc_host->cg.action, &c->sc->cg.action, sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    *action = c->sc_host->cg.action;
    return GPAIR_OK;
}

// One CG run in three phases, so that several contexts can have their runs in
// flight at once (gpair_cg_run_many): prepare (parameters, controller reset,
// graph build, start event), launch, finish (end event, wait, results).
struct CgRun {
    cudaEvent_t e0, e1;
    long long launches0;
    int want_trace;
};

static int cg_validate(gpair_ctx *c, const gpair_cg_params *p)
{
    if (!c || !p || !c->have_problem) return GPAIR_ERR_STATE;
    if (p->iterations < 0 || p->method < 0 || p->method > 4) return GPAIR_ERR_INVALID;
    if (p->line_search != GPAIR_LS_WOLFE && p->line_search != GPAIR_LS_BATCH) return GPAIR_ERR_INVALID;
    if (!(p->target_J >= 0.0)) return GPAIR_ERR_INVALID;
    return GPAIR_OK;
}

static int cg_prepare(gpair_ctx *c, const gpair_cg_params *p, int want_trace, CgRun *r, int build_graph = 1)
{
    int rc = cg_validate(c, p);
    if (rc) return rc;
    GP_CUDA(c, cudaSetDevice(c->device));
    c->fuse_ctrl = -1;
    c->fuse_handles = 0;
    // parameters into the device state
    CgState h;
    memset(&h, 0, sizeof(h));
    h.method = p->method;
    c->cg_method = p->method;
    if (p->method == 4 && (rc = gp_lbfgs_alloc(c))) return rc;
    h.max_zoom = p->max_zoom > 0 ? p->max_zoom : 200;
    h.max_bracket = p->max_bracket > 0 ? p->max_bracket : 100;
    h.alpha = p->alpha;
    h.minvalue = p->minvalue;
    h.c1 = p->wolfe1;
    h.c2 = p->wolfe2;
    h.step_max = p->step_max;
    h.run_limit = p->iterations;
    h.ls_mode = p->line_search;
    h.target_J = p->target_J;
    h.batch_step_max = p->batch_step_max > 0.0 ? p->batch_step_max : 1e12;
    // stop flag shared with racing runs (device pointer or null)
    GP_CUDA(c, cudaMemcpyAsync(&c->sc->stop_flag, &p->stop_flag, sizeof(int *), cudaMemcpyHostToDevice, c->stream));
    if (h.ls_mode == GPAIR_LS_BATCH && (rc = gp_batch_alloc(c))) return rc;
    if (p->resume) {
        // parameters only; the iteration state of the previous run is kept
        GP_CUDA(c, cudaMemcpyAsync(&c->sc->cg, &h, offsetof(CgState, it), cudaMemcpyHostToDevice, c->stream));
        if ((rc = gp_cg_kernel(c, CTRL_RESUME))) return rc;
    } else {
        GP_CUDA(c, cudaMemcpyAsync(&c->sc->cg, &h, sizeof(CgState), cudaMemcpyHostToDevice, c->stream));
        if ((rc = gp_cg_kernel(c, CTRL_INIT))) return rc;
    }
    c->st_n = 0;
    r->want_trace = want_trace;
    r->launches0 = c->launches;
    if (!p->host_loop && build_graph) {
        // build (or reuse) the graph before the timed region
        long long dummy = 0;
        if ((rc = gp_cg_graph_run(c, 0, want_trace, p->line_search, &dummy))) return rc;
        if (c->stage_timing) c->st_n = 0;
    }
    GP_CUDA(c, cudaEventCreate(&r->e0));
    if (cudaEventCreate(&r->e1) != cudaSuccess) {
        cudaEventDestroy(r->e0);
        snprintf(c->last_error, sizeof(c->last_error), "cudaEventCreate failed");
        return GPAIR_ERR_CUDA;
    }
    if (cudaEventRecord(r->e0, c->stream) != cudaSuccess) {
        cudaEventDestroy(r->e0);
        cudaEventDestroy(r->e1);
        snprintf(c->last_error, sizeof(c->last_error), "cudaEventRecord failed");
        return GPAIR_ERR_CUDA;
    }
    return GPAIR_OK;
}

// host-driven iterations (host_loop = 1): the controller's decision is read after every trial
static int cg_host_loop(gpair_ctx *c, const gpair_cg_params *p, double *tJ, double *tchi2, double *tS, double *tstep,
                        double *tbeta, int *it_out)
{
    int status = GPAIR_OK, rc, it = 0;
    for (it = 0; it < p->iterations && status == GPAIR_OK; it++) {
        // the controller steps run in the last block of the preceding reduction kernel
        if ((rc = gp_eval_criterion(c, GPAIR_IMG_CURR, 0))) { status = rc; break; }
        c->fuse_ctrl = CTRL_BEGIN;
        if ((rc = gp_eval_gradient(c, GPAIR_IMG_CURR, -1.f))) { status = rc; break; }
        c->fuse_ctrl = CTRL_AFTER_DIR;
        if ((rc = p->method == 4 ? gp_lbfgs_direction(c) : gp_descent_dir(c, 1, 0.0))) { status = rc; break; }
        int action = CG_EVAL_CRIT, trials = 0;
        if ((rc = read_action(c, &action))) { status = rc; break; }
        while (action != CG_DONE) {
            if (++trials > 10000) { status = GPAIR_ERR_TIMEOUT; break; }
            if (action == CG_EVAL_BATCH) {
                c->fuse_ctrl = CTRL_AFTER_BATCH;
                rc = gp_eval_batch(c);
            } else if (action == CG_EVAL_CRIT) {
                c->fuse_ctrl = CTRL_AFTER_CRIT;
                rc = gp_eval_criterion(c, GPAIR_IMG_TEMP, 1);
            } else {
                c->fuse_ctrl = CTRL_AFTER_GRAD;
                rc = gp_eval_gradient(c, GPAIR_IMG_TEMP, -1.f);
            }
            if (rc) { status = rc; break; }
            if ((rc = read_action(c, &action))) { status = rc; break; }
        }
        if (status) break;
        if ((rc = gp_update_image(c, 1, 0.0, p->minvalue, 1)) || (rc = gp_cg_kernel(c, CTRL_END))) {
            status = rc;
            break;
        }
        if (tJ || tchi2 || tS || tstep || tbeta || it == p->iterations - 1 || p->target_J > 0.0 || p->stop_flag) {
            if ((rc = gp_sync_scalars(c))) { status = rc; break; }
            const CgState &s = c->sc_host->cg;
            if (tJ) tJ[it] = s.J;
            if (tchi2) tchi2[it] = s.chi2;
            if (tS) tS[it] = s.entropy;
            if (tstep) tstep[it] = s.sel;
            if (tbeta) tbeta[it] = s.beta;
            if (c->sc_host->nonfinite) { status = GPAIR_ERR_NUMERIC; it++; break; }
            if (s.reached || s.stopped) { it++; break; }
        }
    }
    *it_out = it;
    return status;
}

static void cg_mark_end(gpair_ctx *c, CgRun *r) { cudaEventRecord(r->e1, c->stream); }

static int cg_finish(gpair_ctx *c, const gpair_cg_params *p, gpair_cg_result *res, double *tJ, double *tchi2,
                     double *tS, double *tstep, double *tbeta, CgRun *r, int status, int it,
                     void *batch_graph = nullptr, int batch_index = 0)
{
    cudaError_t e = cudaEventSynchronize(r->e1);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, r->e0, r->e1);
    cudaEventDestroy(r->e0);
    cudaEventDestroy(r->e1);
    if (e != cudaSuccess) {
        snprintf(c->last_error, sizeof(c->last_error), "CG run: %s", cudaGetErrorString(e));
        return GPAIR_ERR_CUDA;
    }
    if (c->stage_timing) stage_collect(c);
    int rc2 = gp_sync_scalars(c);
    if (rc2 && !status) status = rc2;
    const CgState &s = c->sc_host->cg;
    if (!p->host_loop) {
        it = s.run_it;
        if (r->want_trace && !status && !batch_graph) status = gp_cg_graph_trace(c, it, tJ, tchi2, tS, tstep, tbeta);
        if (!status && c->sc_host->nonfinite) status = GPAIR_ERR_NUMERIC;
        c->launches = r->launches0 + (batch_graph ? gp_batch_graph_launches(batch_graph, batch_index, it,
                                                                            s.criterion_evals, s.grad_evals,
                                                                            s.batches)
                                                  : gp_cg_graph_launches(c, it, s.criterion_evals, s.grad_evals,
                                                                         s.batches));
    }
    c->last_ms = ms;
    double per = 4.0 * (double)c->npix * c->nuv + 8.0 * c->N * (double)c->nuv;
    c->last_flops = per * (s.criterion_evals + s.grad_evals);
    c->last_launches = c->launches - r->launches0;
    if (res) {
        res->iterations_done = it;
        res->criterion_evals = s.criterion_evals;
        res->grad_evals = s.grad_evals;
        res->J = s.J;
        res->chi2 = s.chi2;
        res->entropy = s.entropy;
        res->last_step = s.sel;
        res->last_beta = s.beta;
        res->status = status;
        res->reached = s.reached;
        res->stopped = s.stopped;
    }
    return status;
}

extern "C" int gpair_cg_run(gpair_ctx *c, const gpair_cg_params *p, gpair_cg_result *res, double *tJ, double *tchi2,
                            double *tS, double *tstep, double *tbeta)
{
    CgRun r;
    int rc = cg_prepare(c, p, tJ || tchi2 || tS || tstep || tbeta, &r);
    if (rc) return rc;
    int status, it = 0;
    if (!p->host_loop) {
        long long dummy = 0;
        status = gp_cg_graph_run(c, p->iterations, r.want_trace, p->line_search, &dummy);
    } else {
        status = cg_host_loop(c, p, tJ, tchi2, tS, tstep, tbeta, &it);
    }
    cg_mark_end(c, &r);
    return cg_finish(c, p, res, tJ, tchi2, tS, tstep, tbeta, &r, status, it);
}

// ------------------------------------------------------- batched contexts

struct gpair_batch {
    int n, ls_mode, device;
    gpair_ctx **ctx;
    void *graph;
    cudaStream_t stream;
    cudaEvent_t *ready;
    cudaEvent_t done, e0, e1;
};

extern "C" int gpair_batch_destroy(gpair_batch *b)
{
    if (!b) return GPAIR_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    gp_batch_graph_free(b->graph);
    if (b->ready)
        for (int i = 0; i < b->n; i++)
            if (b->ready[i]) cudaEventDestroy(b->ready[i]);
    if (b->done) cudaEventDestroy(b->done);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    free(b->ready);
    free(b->ctx);
    free(b);
    return GPAIR_OK;
}

extern "C" int gpair_batch_create(gpair_batch **out, gpair_ctx **ctx, int n, int line_search)
{
    return gpair_batch_create_ex(out, ctx, n, line_search, 0);
}

extern "C" int gpair_batch_grouped(const gpair_batch *b) { return b ? gp_batch_graph_grouped(b->graph) : 0; }
extern "C" int gpair_batch_prep_passes(const gpair_batch *b) { return b ? gp_batch_graph_prep_passes(b->graph) : 0; }

extern "C" int gpair_batch_stage_stamps(const gpair_batch *b, unsigned long long *ns, int max, int reset)
{
    if (!b || (!ns && max > 0)) return GPAIR_ERR_INVALID;
    if (cudaSetDevice(b->device) != cudaSuccess) return GPAIR_ERR_CUDA;
    return gp_batch_graph_stamps(b->graph, ns, max, b->stream, reset);
}

extern "C" int gpair_batch_create_ex(gpair_batch **out, gpair_ctx **ctx, int n, int line_search, int flags)
{
    if (!out || !ctx || n <= 0) return GPAIR_ERR_INVALID;
    if (flags & ~(GPAIR_BATCH_INDEPENDENT | GPAIR_BATCH_FORWARDS_ONLY | GPAIR_BATCH_STAGE_STAMPS | (63 << 8)))
        return GPAIR_ERR_INVALID;
    const int prep_passes = (flags >> 8) & 63;  // GPAIR_BATCH_PREP_PASSES(p); 0: chosen by the batch
    if (prep_passes & (prep_passes - 1)) return GPAIR_ERR_INVALID;
    if (line_search != GPAIR_LS_WOLFE && line_search != GPAIR_LS_BATCH) return GPAIR_ERR_INVALID;
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        if (!ctx[i] || !ctx[i]->have_problem || !ctx[i]->have_image) return GPAIR_ERR_STATE;
        if (ctx[i]->device != ctx[0]->device) return GPAIR_ERR_INVALID;
        for (int j = 0; j < i; j++)
            if (ctx[i] == ctx[j]) return GPAIR_ERR_INVALID;
    }
    gpair_batch *b = (gpair_batch *)calloc(1, sizeof(gpair_batch));
    if (!b) return GPAIR_ERR_ALLOC;
    b->n = n;
    b->ls_mode = line_search;
    b->device = ctx[0]->device;
    b->ctx = (gpair_ctx **)calloc((size_t)n, sizeof(gpair_ctx *));
    b->ready = (cudaEvent_t *)calloc((size_t)n, sizeof(cudaEvent_t));
    if (!b->ctx || !b->ready) {
        gpair_batch_destroy(b);
        return GPAIR_ERR_ALLOC;
    }
    memcpy(b->ctx, ctx, sizeof(gpair_ctx *) * n);
    int rc = GPAIR_OK;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) || cudaEventCreate(&b->e0) ||
        cudaEventCreate(&b->e1))
        rc = GPAIR_ERR_CUDA;
    for (int i = 0; i < n && !rc; i++)
        if (cudaEventCreateWithFlags(&b->ready[i], cudaEventDisableTiming) != cudaSuccess) rc = GPAIR_ERR_CUDA;
    for (int i = 0; i < n && !rc; i++) {
        ctx[i]->fuse_ctrl = -1;
        ctx[i]->fuse_handles = 0;
    }
    // 2: every stage grouped where the instances allow it, 1: grouped forwards only, 0: independent
    int group = (flags & GPAIR_BATCH_INDEPENDENT) ? 0 : (flags & GPAIR_BATCH_FORWARDS_ONLY) ? 1 : 2;
    if (flags & GPAIR_BATCH_STAGE_STAMPS) group |= 4;  // device timer stamps between the staged launches
    group |= prep_passes << 8;
    if (!rc) rc = gp_batch_graph_build(ctx, n, line_search, group, &b->graph);
    if (rc) {
        gpair_batch_destroy(b);
        return rc;
    }
    *out = b;
    return GPAIR_OK;
}

extern "C" int gpair_batch_run(gpair_batch *b, const gpair_cg_params *p, gpair_cg_result *res)
{
    if (!b || !p) return GPAIR_ERR_INVALID;
    // the batch graph holds the CG direction update; projected L-BFGS runs per context
    if (p->host_loop || p->line_search != b->ls_mode || p->method == 4) return GPAIR_ERR_INVALID;
    for (int i = 0; i < b->n; i++) {
        int rc = cg_validate(b->ctx[i], p);
        if (rc) return rc;
        // the batch graph was captured with each context's precision path and buffers
        if (gp_batch_graph_precision(b->graph, i) != b->ctx[i]->precision ||
            gp_batch_graph_buf_gen(b->graph, i) != b->ctx[i]->buf_gen)
            return GPAIR_ERR_STATE;
    }
    std::vector<CgRun> r((size_t)b->n);
    GP_CUDA(b->ctx[0], cudaSetDevice(b->device));
    int prepared = 0, rc = GPAIR_OK;
    for (; prepared < b->n; prepared++) {
        gpair_ctx *c = b->ctx[prepared];
        if ((rc = cg_prepare(c, p, 0, &r[prepared], 0))) break;
        cudaEventRecord(b->ready[prepared], c->stream);
        cudaStreamWaitEvent(b->stream, b->ready[prepared], 0);
    }
    float ms = 0.f;
    if (!rc) {
        cudaEventRecord(b->e0, b->stream);
        rc = gp_batch_graph_launch(b->graph, b->stream);
        cudaEventRecord(b->e1, b->stream);
        cudaEventRecord(b->done, b->stream);
        if (!rc && cudaEventSynchronize(b->e1) == cudaSuccess) cudaEventElapsedTime(&ms, b->e0, b->e1);
    }
    int first_err = rc;
    for (int i = 0; i < prepared; i++) {
        gpair_ctx *c = b->ctx[i];
        if (rc) {
            cudaEventDestroy(r[i].e0);
            cudaEventDestroy(r[i].e1);
            continue;
        }
        cudaStreamWaitEvent(c->stream, b->done, 0);
        cg_mark_end(c, &r[i]);
        int rci = cg_finish(c, p, res ? &res[i] : nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &r[i],
                            GPAIR_OK, 0, b->graph, i);
        c->last_ms = ms;
        if (rci && !first_err) first_err = rci;
    }
    return first_err;
}

extern "C" int gpair_cg_run_many(gpair_ctx **ctx, int n, const gpair_cg_params *p, gpair_cg_result *res)
{
    if (!ctx || !p || n <= 0 || p->host_loop) return GPAIR_ERR_INVALID;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++)
            if (ctx[i] == ctx[j]) return GPAIR_ERR_INVALID;  // each run needs its own context and stream
    for (int i = 0; i < n; i++) {
        int rc = cg_validate(ctx[i], p);
        if (rc) return rc;
    }
    CgRun *r = (CgRun *)calloc((size_t)n, sizeof(CgRun));
    int *st = (int *)calloc((size_t)n, sizeof(int));
    if (!r || !st) {
        free(r);
        free(st);
        return GPAIR_ERR_ALLOC;
    }
    int first_err = GPAIR_OK, prepared = 0;
    // every run is prepared (graphs built) before any is launched: a graph
    // capture must not overlap another context's work on the legacy stream
    for (; prepared < n; prepared++) {
        int rc = cg_prepare(ctx[prepared], p, 0, &r[prepared]);
        if (rc) {
            first_err = rc;
            break;
        }
    }
    if (!first_err) {
        for (int i = 0; i < n; i++) {
            long long dummy = 0;
            st[i] = gp_cg_graph_run(ctx[i], p->iterations, 0, p->line_search, &dummy);
            cg_mark_end(ctx[i], &r[i]);
        }
    }
    for (int i = 0; i < prepared; i++) {
        if (first_err) {
            cudaEventDestroy(r[i].e0);
            cudaEventDestroy(r[i].e1);
            continue;
        }
        int rc = cg_finish(ctx[i], p, res ? &res[i] : nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, &r[i],
                           st[i], 0);
        if (rc && !first_err) first_err = rc;
    }
    free(r);
    free(st);
    return first_err;
}

extern "C" int gpair_last_run_stats(gpair_ctx *c, double *ms, double *flops, int *launches)
{
    if (!c) return GPAIR_ERR_INVALID;
    if (ms) *ms = c->last_ms;
    if (flops) *flops = c->last_flops;
    if (launches) *launches = (int)c->last_launches;
    return GPAIR_OK;
}

extern "C" int gpair_time_stages(gpair_ctx *c, int reps, double *ms, int max_stages)
{
    if (!c || !c->have_problem || reps <= 0 || !ms) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    const int ns = GPAIR_NSTAGES;
    std::vector<cudaEvent_t> ev((size_t)(ns + 1) * reps);
    for (auto &e : ev) GP_CUDA(c, cudaEventCreate(&e));
    const bool tc = c->precision != GPAIR_PREC_FP32;
    int rc = GPAIR_OK;
    for (int r = 0; r < reps && !rc; r++) {
        // stages queued back to back: the events time kernels, not host launch gaps
        cudaEvent_t *E = &ev[(size_t)r * (ns + 1)];
        cudaEventRecord(E[0], c->stream);
        if ((rc = tc ? gp_tc_prep_image(c, GPAIR_IMG_CURR) : gp_prep_image(c, GPAIR_IMG_CURR, 0, 0.0, 0))) break;
        cudaEventRecord(E[1], c->stream);
        if ((rc = tc ? gp_tc_forward_gemm(c) : gp_forward(c, GPAIR_IMG_CURR))) break;
        cudaEventRecord(E[2], c->stream);
        if ((rc = gp_vis_data(c))) break;
        cudaEventRecord(E[3], c->stream);
        if ((rc = gp_adj_weights_only(c))) break;
        if (tc && (rc = gp_tc_build_w(c))) break;
        cudaEventRecord(E[4], c->stream);
        if ((rc = tc ? gp_tc_adjoint_gemm(c) : gp_adjoint_contraction(c, GPAIR_IMG_CURR))) break;
        cudaEventRecord(E[5], c->stream);
        if ((rc = gp_grad_finalize(c, GPAIR_IMG_CURR, GRAD_FUSED, 1e-3f))) break;
        cudaEventRecord(E[6], c->stream);
    }
    double acc[GPAIR_NSTAGES] = {0};
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GPAIR_ERR_CUDA;
    for (int r = 0; r < reps && !rc; r++) {
        cudaEvent_t *E = &ev[(size_t)r * (ns + 1)];
        for (int i = 0; i < ns; i++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, E[i], E[i + 1]);
            acc[i] += t;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    int n = max_stages < ns ? max_stages : ns;
    for (int i = 0; i < n; i++) ms[i] = acc[i] / reps;
    return n;
}

// The three stages of one batched line-search evaluation (8 trial images), timed
// like gpair_time_stages: [0] trial images + operands, [1] forward contraction
// of the stack, [2] chi2 of every trial. The steps are the device state's last
// batch (or the initial grid); the controller does not run.
extern "C" int gpair_time_batch_stages(gpair_ctx *c, int reps, double *ms, int max_stages)
{
    if (!c || !c->have_problem || reps <= 0 || !ms) return GPAIR_ERR_INVALID;
    GP_CUDA(c, cudaSetDevice(c->device));
    int rc = gp_batch_alloc(c);
    if (rc) return rc;
    const int ns = 3;
    std::vector<cudaEvent_t> ev((size_t)(ns + 1) * reps);
    for (auto &e : ev) GP_CUDA(c, cudaEventCreate(&e));
    const int st = c->stage_timing;
    c->stage_timing = 0;
    for (int r = 0; r < reps && !rc; r++) {
        cudaEvent_t *E = &ev[(size_t)r * (ns + 1)];
        c->fuse_ctrl = -1;
        rc = gp_eval_batch_timed(c, E);
    }
    c->stage_timing = st;
    double acc[3] = {0, 0, 0};
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = GPAIR_ERR_CUDA;
    for (int r = 0; r < reps && !rc; r++) {
        cudaEvent_t *E = &ev[(size_t)r * (ns + 1)];
        for (int i = 0; i < ns; i++) {
            float t = 0.f;
            cudaEventElapsedTime(&t, E[i], E[i + 1]);
            acc[i] += t;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    int n = max_stages < ns ? max_stages : ns;
    for (int i = 0; i < n; i++) ms[i] = acc[i] / reps;
    return n;
}
