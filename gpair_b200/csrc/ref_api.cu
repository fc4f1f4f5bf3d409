// ref_api.cu -- the reference's GPU boundary (gpair1/trunk/gpu.h:5-120) on
// top of the B200 context.
//
// Same names, argument order and meaning as gpair1/trunk/gpu.c. Like the
// reference these calls use one global context, block until the device work
// is finished, and on failure print a message and exit(0)
// (print_opencl_error, gpair1/trunk/gpu.c:186-202); gpair_set_exit_on_error(0)
// makes them print and return instead (tests use this).
//
// The reference uploads data before it knows nuv / nbis (those arrive with
// every gpu_get_chi2 call), so gpu_copy_data and gpu_copy_dft stage the
// caller's arrays on the host and the problem is bound to the device at the
// first call that carries (nuv, npow, nbis) -- and rebound if they change.
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "gpair_internal.cuh"

int gp_alloc_images(gpair_ctx *c, int N);
int gp_set_problem_core(gpair_ctx *c, int N, float pix, int nuv, const gpair_uv *uv, int npow, int nbis,
                        const float *data, const float *data_err, const gpair_float2 *phasor, const int64_t *uvpnt,
                        const int16_t *sign, const float *model);
int gp_eval_criterion(gpair_ctx *c, int which, int trial);

static gpair_ctx *g_ctx = nullptr;
static int g_exit_on_error = 1;

extern "C" void gpair_set_exit_on_error(int on) { g_exit_on_error = on; }
extern "C" gpair_ctx *gpair_global_context(void) { return g_ctx; }

extern "C" char *print_cl_errstring(int err) { return (char *)gpair_strerror(err); }

extern "C" void print_opencl_error(char *error_message, int error_code)
{
    printf("GPU Error: %s\nError code: %d (%s)\n", error_message ? error_message : "", error_code,
           gpair_strerror(error_code));
    if (g_ctx && g_ctx->last_error[0]) printf("Detail: %s\n", g_ctx->last_error);
    fflush(stdout);
    if (g_exit_on_error) {
        gpu_cleanup();
        exit(0);
    }
}

extern "C" int gpu_error_callback(char *error)
{
    printf("Callback function called!\n %s", error);
    return 0;
}

#define REF_CHECK(expr, msg)                                   \
    do {                                                       \
        int rc_ = (expr);                                      \
        if (rc_ != GPAIR_OK) {                                 \
            print_opencl_error((char *)(msg), rc_);            \
            return;                                            \
        }                                                      \
    } while (0)
#define REF_CHECK_V(expr, msg, val)                            \
    do {                                                       \
        int rc_ = (expr);                                      \
        if (rc_ != GPAIR_OK) {                                 \
            print_opencl_error((char *)(msg), rc_);            \
            return (val);                                      \
        }                                                      \
    } while (0)

static int need_ctx(void) { return g_ctx ? GPAIR_OK : GPAIR_ERR_STATE; }

static int which_of(gpair_buf *b)
{
    if (b && g_ctx && b->ptr == g_ctx->image_temp) return GPAIR_IMG_TEMP;
    return GPAIR_IMG_CURR;
}

// Bind the staged arrays for (nuv, npow, nbis); no-op when already bound.
static int bind(int nuv, int npow, int nbis)
{
    gpair_ctx *c = g_ctx;
    if (!c) return GPAIR_ERR_STATE;
    if (c->have_problem && c->bound_nuv == nuv && c->bound_npow == npow && c->bound_nbis == nbis) return GPAIR_OK;
    if (!c->ref_data || !c->ref_dft_x) {
        snprintf(c->last_error, sizeof(c->last_error), "gpu_copy_data and gpu_copy_dft must precede evaluation");
        return GPAIR_ERR_STATE;
    }
    long long nd = npow + 2LL * nbis;
    if (npow != c->ref_npow || nd > c->ref_data_size || nbis > c->ref_bsref_size || nbis > c->ref_phasor_size
        || (long long)nuv * c->N > c->ref_dft_size || npow > nuv) {
        snprintf(c->last_error, sizeof(c->last_error), "sizes (nuv %d npow %d nbis %d) exceed the uploaded arrays", nuv,
                 npow, nbis);
        return GPAIR_ERR_INVALID;
    }
    std::vector<int64_t> uvpnt((size_t)3 * nbis);
    std::vector<int16_t> sign((size_t)3 * nbis);
    for (int t = 0; t < nbis; t++) {
        uvpnt[3 * t] = c->ref_uvpnt[t].s0;
        uvpnt[3 * t + 1] = c->ref_uvpnt[t].s1;
        uvpnt[3 * t + 2] = c->ref_uvpnt[t].s2;
        sign[3 * t] = c->ref_sign[t].s0;
        sign[3 * t + 1] = c->ref_sign[t].s1;
        sign[3 * t + 2] = c->ref_sign[t].s2;
    }
    int rc = gp_set_problem_core(c, c->N, 0.f, nuv, nullptr, npow, nbis, c->ref_data, c->ref_data_err,
                                 c->ref_phasor, uvpnt.data(), sign.data(), c->ref_model);
    if (rc) return rc;
    rc = gp_twiddles_from_ref_tables(c, (const float2 *)c->ref_dft_x, (const float2 *)c->ref_dft_y);
    if (rc) return rc;
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->bound_nuv = nuv;
    c->bound_npow = npow;
    c->bound_nbis = nbis;
    return GPAIR_OK;
}

static int sync_ctx(void)
{
    GP_CUDA(g_ctx, cudaStreamSynchronize(g_ctx->stream));
    return GPAIR_OK;
}

// ------------------------------------------------------------- lifecycle

extern "C" void gpu_init(void)
{
    if (g_ctx) gpu_cleanup();
    int dev = 0;
    const char *e = getenv("GPAIR_DEVICE");
    if (e) dev = atoi(e);
    int rc = gpair_create(&g_ctx, dev);
    if (rc) {
        g_ctx = nullptr;
        print_opencl_error((char *)"Failed to create a device context.", rc);
    }
}

extern "C" void gpu_cleanup(void)
{
    if (g_ctx) gpair_destroy(g_ctx);
    g_ctx = nullptr;
}

extern "C" void gpu_shutdown(void) { gpu_cleanup(); }

extern "C" void gpu_build_kernels(int data_size, int image_width, int image_size)
{
    (void)data_size;
    REF_CHECK(need_ctx(), "gpu_build_kernels before gpu_init");
    if (image_width != g_ctx->N || image_size != g_ctx->npix)
        print_opencl_error((char *)"gpu_build_kernels: image size differs from gpu_copy_data", GPAIR_ERR_INVALID);
}

// ------------------------------------------------------------ uploads

extern "C" void gpu_copy_data(float *data, float *data_err, int data_size, int data_size_uv, gpair_float2 *data_phasor,
                              int phasor_size, int pow_size, gpair_long4 *uvpnt, gpair_short4 *sign, int bsref_size,
                              float *default_model, int image_size, int image_width)
{
    (void)data_size_uv;
    REF_CHECK(need_ctx(), "gpu_copy_data before gpu_init");
    gpair_ctx *c = g_ctx;
    if (image_width <= 0 || image_size != image_width * image_width || data_size < pow_size || data_size < 0) {
        print_opencl_error((char *)"gpu_copy_data: inconsistent sizes", GPAIR_ERR_INVALID);
        return;
    }
    REF_CHECK(gp_alloc_images(c, image_width), "Could not allocate image buffers.");
    free(c->ref_data); free(c->ref_data_err); free(c->ref_model); free(c->ref_phasor); free(c->ref_uvpnt); free(c->ref_sign);
    c->ref_data = (float *)malloc(sizeof(float) * (data_size + 1));
    c->ref_data_err = (float *)malloc(sizeof(float) * (data_size + 1));
    c->ref_model = (float *)malloc(sizeof(float) * image_size);
    c->ref_phasor = (gpair_float2 *)malloc(sizeof(gpair_float2) * (phasor_size + 1));
    c->ref_uvpnt = (gpair_long4 *)malloc(sizeof(gpair_long4) * (bsref_size + 1));
    c->ref_sign = (gpair_short4 *)malloc(sizeof(gpair_short4) * (bsref_size + 1));
    memcpy(c->ref_data, data, sizeof(float) * data_size);
    memcpy(c->ref_data_err, data_err, sizeof(float) * data_size);
    memcpy(c->ref_model, default_model, sizeof(float) * image_size);
    if (phasor_size) memcpy(c->ref_phasor, data_phasor, sizeof(gpair_float2) * phasor_size);
    if (bsref_size) {
        memcpy(c->ref_uvpnt, uvpnt, sizeof(gpair_long4) * bsref_size);
        memcpy(c->ref_sign, sign, sizeof(gpair_short4) * bsref_size);
    }
    c->ref_data_size = data_size;
    c->ref_phasor_size = phasor_size;
    c->ref_bsref_size = bsref_size;
    c->ref_npow = pow_size;
    c->have_problem = 0;
    // the reference zeroes the gradient buffers and images here (gpu.c:1317-1345)
    size_t bytes = sizeof(float) * c->npix;
    float *zero_bufs[] = {c->image, c->image_temp, c->data_grad, c->entropy_grad, c->full_grad_new,
                          c->full_grad, c->grad_temp, c->descent_dir};
    for (float *b : zero_bufs) REF_CHECK(cudaMemsetAsync(b, 0, bytes, c->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA,
                                         "Could not clear device buffers.");
    REF_CHECK(cudaMemcpyAsync(c->model, default_model, bytes, cudaMemcpyHostToDevice, c->stream) == cudaSuccess
                  ? 0 : GPAIR_ERR_CUDA, "Could not copy the default model.");
    REF_CHECK(sync_ctx(), "gpu_copy_data");
}

extern "C" void gpu_copy_dft(gpair_float2 *dft_x, gpair_float2 *dft_y, int dft_size)
{
    REF_CHECK(need_ctx(), "gpu_copy_dft before gpu_init");
    gpair_ctx *c = g_ctx;
    free(c->ref_dft_x);
    free(c->ref_dft_y);
    c->ref_dft_x = (gpair_float2 *)malloc(sizeof(gpair_float2) * (dft_size + 1));
    c->ref_dft_y = (gpair_float2 *)malloc(sizeof(gpair_float2) * (dft_size + 1));
    memcpy(c->ref_dft_x, dft_x, sizeof(gpair_float2) * dft_size);
    memcpy(c->ref_dft_y, dft_y, sizeof(gpair_float2) * dft_size);
    c->ref_dft_size = dft_size;
    c->have_problem = 0;
}

extern "C" void gpu_copy_image(float *image, int x_size, int y_size)
{
    REF_CHECK(need_ctx(), "gpu_copy_image before gpu_init");
    if (x_size * y_size != g_ctx->npix) {
        print_opencl_error((char *)"Error copying image to the GPU", GPAIR_ERR_INVALID);
        return;
    }
    REF_CHECK(gpair_set_image(g_ctx, GPAIR_IMG_CURR, image), "Error copying image to the GPU");
}

// ------------------------------------------------------------ criterion

extern "C" void gpu_image2vis(int nuv, int data_alloc_uv, gpair_buf *gpu_image)
{
    (void)data_alloc_uv;
    REF_CHECK(need_ctx(), "Invalid Image, did you forget to initalize?");
    REF_CHECK(gpu_image ? 0 : GPAIR_ERR_INVALID, "Invalid Image, did you forget to initalize?");
    gpair_ctx *c = g_ctx;
    int npow = c->have_problem ? c->bound_npow : c->ref_npow;
    int nbis = c->have_problem ? c->bound_nbis : 0;
    if (!c->have_problem || c->bound_nuv != nuv) REF_CHECK(bind(nuv, npow, nbis), "Cannot bind the problem.");
    int w = which_of(gpu_image);
    REF_CHECK(gp_prep_image(c, w, 0, 0.0, 0), "Cannot compute the flux.");
    REF_CHECK(gp_forward(c, w), "Cannot Enqueue visi kernel.");
    // visibilities (with 1/F) are formed by the data kernel; run it now so that
    // the stored visibilities are complete after this call
    REF_CHECK(gp_vis_data(c), "Cannot Enqueue visi kernel.");
    c->last_image_src = w;
    REF_CHECK(sync_ctx(), "gpu_image2vis");
}

extern "C" void gpu_vis2data(gpair_buf *gpu_vis, int nuv, int npow, int nbis)
{
    (void)gpu_vis;
    REF_CHECK(bind(nuv, npow, nbis), "Cannot bind the problem.");
    REF_CHECK(gp_vis_data(g_ctx), "Could not enqueue bispectrum visi kernel.");
    REF_CHECK(sync_ctx(), "gpu_vis2data");
}

extern "C" void gpu_data2chi2(int data_size)
{
    (void)data_size;  // chi2 is reduced by the data kernel; nothing left to do
    REF_CHECK(need_ctx(), "gpu_data2chi2 before gpu_init");
    REF_CHECK(sync_ctx(), "gpu_data2chi2");
}

extern "C" void gpu_new_chi2(int nuv, int npow, int nbis, int data_alloc)
{
    (void)data_alloc;
    gpu_vis2data(nullptr, nuv, npow, nbis);
}

extern "C" void gpu_image2chi2(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, gpair_buf *gpu_image)
{
    (void)data_alloc; (void)data_alloc_uv;
    REF_CHECK(bind(nuv, npow, nbis), "Cannot bind the problem.");
    REF_CHECK(gpu_image ? 0 : GPAIR_ERR_INVALID, "Image for computing image2chi2 is NULL!");
    REF_CHECK(gp_eval_criterion(g_ctx, which_of(gpu_image), 0), "gpu_image2chi2");
    REF_CHECK(sync_ctx(), "gpu_image2chi2");
}

extern "C" float gpu_get_chi2(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, gpair_buf *gpu_image)
{
    gpu_image2chi2(nuv, npow, nbis, data_alloc, data_alloc_uv, gpu_image);
    if (!g_ctx) return 0.f;
    REF_CHECK_V(gp_sync_scalars(g_ctx), "Could not read back chi2 from the GPU!", 0.f);
    return (float)g_ctx->sc_host->chi2;
}

extern "C" float gpu_get_chi2_curr(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv)
{
    REF_CHECK_V(need_ctx(), "gpu_get_chi2_curr before gpu_init", 0.f);
    return gpu_get_chi2(nuv, npow, nbis, data_alloc, data_alloc_uv, &g_ctx->h_image);
}

extern "C" float gpu_get_chi2_temp(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv)
{
    REF_CHECK_V(need_ctx(), "gpu_get_chi2_temp before gpu_init", 0.f);
    return gpu_get_chi2(nuv, npow, nbis, data_alloc, data_alloc_uv, &g_ctx->h_image_temp);
}

extern "C" void gpu_compute_flux(gpair_buf *gpu_image, gpair_buf *flux_storage, gpair_buf *flux_inverse_storage)
{
    REF_CHECK(need_ctx(), "gpu_compute_flux before gpu_init");
    REF_CHECK(gp_prep_image(g_ctx, which_of(gpu_image), 0, 0.0, 0), "Could not compute the flux.");
    gpair_ctx *c = g_ctx;
    if (flux_storage && flux_storage->ptr && flux_storage->count >= 1)
        REF_CHECK(cudaMemcpyAsync(flux_storage->ptr, &c->sc->flux_f, sizeof(float), cudaMemcpyDeviceToDevice,
                                  c->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "Could not read back the flux value.");
    if (flux_inverse_storage && flux_inverse_storage->ptr && flux_inverse_storage->count >= 1)
        REF_CHECK(cudaMemcpyAsync(flux_inverse_storage->ptr, &c->sc->invflux_f, sizeof(float),
                                  cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA,
                  "Could not read back 1/flux.");
    REF_CHECK(sync_ctx(), "gpu_compute_flux");
}

extern "C" void gpu_compute_entropy(int image_width, gpair_buf *gpu_image, gpair_buf *entropy_storage)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_compute_entropy before gpu_init");
    REF_CHECK((gpu_image && entropy_storage) ? 0 : GPAIR_ERR_INVALID, "A pointer to gpu_compute_entropy is NULL!");
    REF_CHECK(gp_prep_image(g_ctx, which_of(gpu_image), 0, 0.0, 0), "Cannot enqueue entropy kernel.");
    if (entropy_storage->ptr && entropy_storage->count >= 1)
        REF_CHECK(cudaMemcpyAsync(entropy_storage->ptr, &g_ctx->sc->entropy_f, sizeof(float),
                                  cudaMemcpyDeviceToDevice, g_ctx->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA,
                  "Cannot store the entropy.");
    REF_CHECK(sync_ctx(), "gpu_compute_entropy");
}

extern "C" float gpu_get_entropy(int image_width, gpair_buf *gpu_image)
{
    (void)image_width;
    REF_CHECK_V(need_ctx(), "gpu_get_entropy before gpu_init", 0.f);
    REF_CHECK_V(gpu_image ? 0 : GPAIR_ERR_INVALID, "Image for computing entropy is NULL!", 0.f);
    REF_CHECK_V(gp_prep_image(g_ctx, which_of(gpu_image), 0, 0.0, 0), "Cannot enqueue entropy kernel.", 0.f);
    REF_CHECK_V(gp_sync_scalars(g_ctx), "Could not read back Entropy from the GPU!", 0.f);
    return (float)g_ctx->sc_host->entropy;
}

extern "C" float gpu_get_entropy_curr(int image_width)
{
    REF_CHECK_V(need_ctx(), "gpu_get_entropy_curr before gpu_init", 0.f);
    return gpu_get_entropy(image_width, &g_ctx->h_image);
}

extern "C" float gpu_get_entropy_temp(int image_width)
{
    REF_CHECK_V(need_ctx(), "gpu_get_entropy_temp before gpu_init", 0.f);
    return gpu_get_entropy(image_width, &g_ctx->h_image_temp);
}

// ------------------------------------------------------------- gradients

extern "C" void gpu_compute_data_gradient(gpair_buf *gpu_image, int nuv, int npow, int nbis, int image_width)
{
    (void)image_width;
    REF_CHECK(gpu_image ? 0 : GPAIR_ERR_INVALID, "Image input is NULL in gpu_compute_data_gradient");
    REF_CHECK(bind(nuv, npow, nbis), "Cannot bind the problem.");
    gpair_ctx *c = g_ctx;
    int w = which_of(gpu_image);
    // the reference recomputes the flux of this image (gpu.c:1607) and uses the
    // visibilities and mock data of the preceding chi2 evaluation
    REF_CHECK(gp_prep_image(c, w, 0, 0.0, 0), "Cannot compute the flux.");
    REF_CHECK(gp_adjoint(c, w), "Cannot enqueue powerspectrum gradient kernel.");
    REF_CHECK(gp_grad_finalize(c, w, GRAD_DATA_ONLY, 0.f), "Cannot enqueue bispectrum gradient kernel.");
    REF_CHECK(sync_ctx(), "gpu_compute_data_gradient");
}

extern "C" void gpu_compute_data_gradient_curr(int nuv, int npow, int nbis, int image_width)
{
    REF_CHECK(need_ctx(), "gpu_compute_data_gradient_curr before gpu_init");
    gpu_compute_data_gradient(&g_ctx->h_image, nuv, npow, nbis, image_width);
}

extern "C" void gpu_compute_data_gradient_temp(int nuv, int npow, int nbis, int image_width)
{
    REF_CHECK(need_ctx(), "gpu_compute_data_gradient_temp before gpu_init");
    gpu_compute_data_gradient(&g_ctx->h_image_temp, nuv, npow, nbis, image_width);
}

extern "C" void gpu_compute_entropy_gradient(int image_width, gpair_buf *gpu_image)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_compute_entropy_gradient before gpu_init");
    REF_CHECK(gpu_image ? 0 : GPAIR_ERR_INVALID, "Pointer to compute_entropy_gradient is NULL!");
    REF_CHECK(gp_entropy_gradient(g_ctx, which_of(gpu_image)), "Cannot enqueue entropy gradient kernel.");
    REF_CHECK(sync_ctx(), "gpu_compute_entropy_gradient");
}

extern "C" void gpu_compute_entropy_gradient_curr(int image_width)
{
    REF_CHECK(need_ctx(), "gpu_compute_entropy_gradient_curr before gpu_init");
    gpu_compute_entropy_gradient(image_width, &g_ctx->h_image);
}

extern "C" void gpu_compute_entropy_gradient_temp(int image_width)
{
    REF_CHECK(need_ctx(), "gpu_compute_entropy_gradient_temp before gpu_init");
    gpu_compute_entropy_gradient(image_width, &g_ctx->h_image_temp);
}

extern "C" void gpu_compute_criterion_gradient(int image_width, float hyperparameter_entropy, gpair_buf *gradient_buffer)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_compute_criterion_gradient before gpu_init");
    REF_CHECK(gradient_buffer ? 0 : GPAIR_ERR_INVALID, "Gradient buffer is NULL.");
    REF_CHECK(gp_criterion_gradient(g_ctx, hyperparameter_entropy, gradient_buffer->ptr),
              "Cannot enqueue Criterion Gradient kernel.");
    REF_CHECK(sync_ctx(), "gpu_compute_criterion_gradient");
}

extern "C" void gpu_compute_criterion_gradient_curr(int image_width, float hyperparameter_entropy)
{
    REF_CHECK(need_ctx(), "gpu_compute_criterion_gradient_curr before gpu_init");
    gpu_compute_criterion_gradient(image_width, hyperparameter_entropy, &g_ctx->h_fgn);
}

extern "C" void gpu_compute_criterion_gradient_temp(int image_width, float hyperparameter_entropy)
{
    REF_CHECK(need_ctx(), "gpu_compute_criterion_gradient_temp before gpu_init");
    gpu_compute_criterion_gradient(image_width, hyperparameter_entropy, &g_ctx->h_tg);
}

// ------------------------------------------------------------ CG vectors

extern "C" void gpu_scalar_prod(int data_width, int data_height, gpair_buf *array1, gpair_buf *array2,
                                gpair_buf *final_output)
{
    REF_CHECK(need_ctx(), "gpu_scalar_prod before gpu_init");
    REF_CHECK((array1 && array2) ? 0 : GPAIR_ERR_INVALID, "Pointer to gpu_sclar_prod is NULL!");
    int n = data_width * data_height;
    if ((size_t)n > array1->count || (size_t)n > array2->count) {
        print_opencl_error((char *)"gpu_scalar_prod: size exceeds the buffers", GPAIR_ERR_INVALID);
        return;
    }
    REF_CHECK(gp_dot(g_ctx, array1->ptr, array2->ptr, n), "Could not enqueue scalar product kernel.");
    if (final_output && final_output->ptr && final_output->count >= 1)
        REF_CHECK(cudaMemcpyAsync(final_output->ptr, &g_ctx->sc->dot_f, sizeof(float), cudaMemcpyDeviceToDevice,
                                  g_ctx->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "Could not store the product.");
    REF_CHECK(sync_ctx(), "gpu_scalar_prod");
}

extern "C" float gpu_get_scalprod(int data_width, int data_height, gpair_buf *array1, gpair_buf *array2)
{
    gpu_scalar_prod(data_width, data_height, array1, array2, nullptr);
    if (!g_ctx) return 0.f;
    REF_CHECK_V(gp_sync_scalars(g_ctx), "Could not read back scalar product value from GPU!", 0.f);
    return g_ctx->sc_host->dot_f;
}

extern "C" void gpu_compute_descent_dir(int image_width, float beta)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_compute_descent_dir before gpu_init");
    REF_CHECK(gp_descent_dir(g_ctx, 0, (double)beta), "Descent Direction Kernel.");
    REF_CHECK(sync_ctx(), "gpu_compute_descent_dir");
}

// float arithmetic of kernel_update_image.cl
__global__ void k_ref_update_image(float *__restrict__ img, const float *__restrict__ d, int n, float s, float minval)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float t = img[p] + s * d[p];
    if (t < minval) t = minval;
    img[p] = t;
}

// float arithmetic of kernel_update_tempimage.cl / kernel_criterion_step.cl
__global__ void k_ref_update_temp(const float *__restrict__ img, const float *__restrict__ d, int n, float s,
                                  float minval, int clamp, float *__restrict__ temp)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float t = img[p] + s * d[p];
    if (clamp && t < minval) t = minval;
    temp[p] = t;
}

extern "C" void gpu_update_image(int image_width, float steplength, float minval, gpair_buf *descent_direction)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_update_image before gpu_init");
    REF_CHECK(descent_direction ? 0 : GPAIR_ERR_INVALID, "Descent Direction to update_image is NULL!");
    gpair_ctx *c = g_ctx;
    k_ref_update_image<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(c->image, descent_direction->ptr, c->npix,
                                                                     steplength, minval);
    REF_CHECK(cudaGetLastError() == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "Cannot enqueue image update kernel.");
    REF_CHECK(sync_ctx(), "gpu_update_image");
}

extern "C" void gpu_update_tempimage(int image_width, float steplength, float minval, gpair_buf *descent_direction)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_update_tempimage before gpu_init");
    REF_CHECK(descent_direction ? 0 : GPAIR_ERR_INVALID, "Descent Direction to update_tempimage is NULL!");
    gpair_ctx *c = g_ctx;
    k_ref_update_temp<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(c->image, descent_direction->ptr, c->npix,
                                                                    steplength, minval, 1, c->image_temp);
    REF_CHECK(cudaGetLastError() == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "Cannot temp image update kernel.");
    REF_CHECK(sync_ctx(), "gpu_update_tempimage");
}

extern "C" void gpu_compute_criterion_step(int image_width, float steplength, float minvalue)
{
    (void)image_width;
    REF_CHECK(need_ctx(), "gpu_compute_criterion_step before gpu_init");
    gpair_ctx *c = g_ctx;
    k_ref_update_temp<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(c->image, c->descent_dir, c->npix, steplength,
                                                                    minvalue, 0, c->image_temp);
    REF_CHECK(cudaGetLastError() == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "Cannot enqueue criterion step kernel.");
    REF_CHECK(sync_ctx(), "gpu_compute_criterion_step");
}

extern "C" void gpu_backup_gradient(int data_size, gpair_buf *input, gpair_buf *output)
{
    REF_CHECK(need_ctx(), "gpu_backup_gradient before gpu_init");
    REF_CHECK((input && output) ? 0 : GPAIR_ERR_INVALID, "Pointer to input or output is NULL in backup_gradient!");
    if ((size_t)data_size > input->count || (size_t)data_size > output->count) {
        print_opencl_error((char *)"gpu_backup_gradient: size exceeds the buffers", GPAIR_ERR_INVALID);
        return;
    }
    REF_CHECK(cudaMemcpyAsync(output->ptr, input->ptr, sizeof(float) * data_size, cudaMemcpyDeviceToDevice,
                              g_ctx->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA, "gpu_backup_gradient");
    REF_CHECK(sync_ctx(), "gpu_backup_gradient");
}

extern "C" float *gpu_get_image(int size, float *cpu_buffer, gpair_buf *gpu_image)
{
    REF_CHECK_V(need_ctx(), "gpu_get_image before gpu_init", cpu_buffer);
    REF_CHECK_V(gpu_image ? 0 : GPAIR_ERR_INVALID, "Could not read back image from the GPU!", cpu_buffer);
    if ((size_t)size > gpu_image->count) {
        print_opencl_error((char *)"Could not read back image from the GPU!", GPAIR_ERR_INVALID);
        return cpu_buffer;
    }
    if (!cpu_buffer) cpu_buffer = (float *)malloc(sizeof(float) * size);  // caller frees
    REF_CHECK_V(cudaMemcpyAsync(cpu_buffer, gpu_image->ptr, sizeof(float) * size, cudaMemcpyDeviceToHost,
                                g_ctx->stream) == cudaSuccess ? 0 : GPAIR_ERR_CUDA,
                "Could not read back image from the GPU!", cpu_buffer);
    REF_CHECK_V(sync_ctx(), "Could not read back image from the GPU!", cpu_buffer);
    return cpu_buffer;
}

extern "C" gpair_buf *gpu_getp_ci(void) { return g_ctx ? &g_ctx->h_image : nullptr; }
extern "C" gpair_buf *gpu_getp_ti(void) { return g_ctx ? &g_ctx->h_image_temp : nullptr; }
extern "C" gpair_buf *gpu_getp_fgn(void) { return g_ctx ? &g_ctx->h_fgn : nullptr; }
extern "C" gpair_buf *gpu_getp_fg(void) { return g_ctx ? &g_ctx->h_fg : nullptr; }
extern "C" gpair_buf *gpu_getp_dd(void) { return g_ctx ? &g_ctx->h_dd : nullptr; }
extern "C" gpair_buf *gpu_getp_tg(void) { return g_ctx ? &g_ctx->h_tg : nullptr; }
extern "C" gpair_buf *gpu_getp_eg(void) { return g_ctx ? &g_ctx->h_eg : nullptr; }

// ------------------------------------------------------------ line search

// The reference's zoom can spin forever once steplength_low and
// steplength_high are adjacent floats far from zero (their difference never
// drops below 1e-14). This one stops after g_zoom_cap trials (200 unless set)
// and returns steplength_low, like the reference's exit with no better point.
// Each stop at the cap is counted and recorded in the global context's
// last_error, so a caller of the drop-in layer can tell.
static int g_zoom_cap = 200;
static int g_zoom_cap_hits = 0;

extern "C" int gpair_set_zoom_trial_cap(int cap)
{
    if (cap < 0) return GPAIR_ERR_INVALID;
    g_zoom_cap = cap ? cap : 200;
    return GPAIR_OK;
}

extern "C" int gpair_zoom_cap_hits(void) { return g_zoom_cap_hits; }

extern "C" void gpair_zoom_cap_hits_reset(void) { g_zoom_cap_hits = 0; }

// gpair1/trunk/gpu.c:1947-2065, float scalars as in the reference. The
// reference's `*criterion_evals++` advances a local pointer and leaves the
// counters untouched; the counters are left untouched here as well.
extern "C" float gpu_linesearch_zoom(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, int image_width,
                                     float steplength_low, float steplength_high, float criterion_steplength_low,
                                     float wolfe_product1, float criterion_init, int *criterion_evals, int *grad_evals,
                                     gpair_buf *pDescent_direction, gpair_buf *pTemp_gradient,
                                     float hyperparameter_entropy)
{
    (void)criterion_evals; (void)grad_evals;
    float chi2, entropy;
    float steplength = 0., selected_steplength = 0., criterion = 0., criterion_old = 0., steplength_old = 0.,
          wolfe_product2;
    int counter = 0;
    float minvalue = 1e-8;
    float wolfe_param1 = 1e-4, wolfe_param2 = 0.1;
    for (int guard = 0; guard < g_zoom_cap; guard++) {
        if ((counter > 0) && (criterion_old - criterion_init - wolfe_product1 * steplength_old) != 0.)
            steplength = fabs(wolfe_product1 * steplength_old * steplength_old
                              / (2. * (criterion_old - criterion_init - wolfe_product1 * steplength_old)));
        if ((counter == 0) || (steplength < steplength_low) || (steplength > steplength_high))
            steplength = (steplength_high - steplength_low) / 2. + steplength_low;
        if (fabs(steplength_high - steplength_low) < 1e-14) return steplength_low;
        gpu_update_tempimage(image_width, steplength, minvalue, pDescent_direction);
        chi2 = gpu_get_chi2_temp(nuv, npow, nbis, data_alloc, data_alloc_uv);
        entropy = gpu_get_entropy_temp(image_width);
        criterion = chi2 - hyperparameter_entropy * entropy;
        if ((criterion > (criterion_init + wolfe_param1 * steplength * wolfe_product1))
            || (criterion >= criterion_steplength_low)) {
            steplength_high = steplength;
        } else {
            gpu_compute_data_gradient_temp(nuv, npow, nbis, image_width);
            gpu_compute_entropy_gradient_temp(image_width);
            gpu_compute_criterion_gradient_temp(image_width, hyperparameter_entropy);
            wolfe_product2 = gpu_get_scalprod(image_width, image_width, pDescent_direction, pTemp_gradient);
            if ((wolfe_product2 >= wolfe_param2 * wolfe_product1) || (counter > 10)) {
                selected_steplength = steplength;
                return selected_steplength;
            }
            if (wolfe_product2 * (steplength_high - steplength_low) >= 0.) steplength_high = steplength_low;
            steplength_low = steplength;
        }
        steplength_old = steplength;
        criterion_old = criterion;
        counter++;
    }
    g_zoom_cap_hits++;
    if (g_ctx)
        snprintf(g_ctx->last_error, sizeof(g_ctx->last_error),
                 "gpu_linesearch_zoom stopped at its %d-trial cap and returned steplength_low %.9g", g_zoom_cap,
                 (double)steplength_low);
    return steplength_low;
}

// -------------------------------------------------------------- debugging

extern "C" void gpu_compare_data(int size, float *cpu_data, gpair_buf *pGpu_data)
{
    if (!g_ctx || !pGpu_data || !cpu_data) return;
    std::vector<float> g(size);
    gpu_get_image(size, g.data(), pGpu_data);
    float max_err = 0.f;
    for (int i = 0; i < size; i++) {
        float err = cpu_data[i] != 0.f ? fabsf((g[i] - cpu_data[i]) / cpu_data[i]) : fabsf(g[i]);
        printf("[%i] CPU %f GPU %f Rel. err %f\n", i, cpu_data[i], g[i], err);
        if (err > max_err) max_err = err;
    }
    printf("Max relative error: %f\n", max_err);
}

extern "C" void gpu_compare_complex_data(int size, float *cpu_data, gpair_buf *pGpu_data)
{
    if (!g_ctx || !pGpu_data || !cpu_data) return;
    std::vector<float> g(2 * (size_t)size);
    gpu_get_image(2 * size, g.data(), pGpu_data);
    float err_sum = 0.f;
    for (int i = 0; i < size; i++) {
        float re = g[2 * i] - cpu_data[2 * i], im = g[2 * i + 1] - cpu_data[2 * i + 1];
        float error = sqrtf(re * re + im * im);
        if (error > 0.01f)
            printf("[%i] %f %f R(A) %f R(B) %f I(A) %f I(B) %f Err: %f\n", i, re, im, cpu_data[2 * i], g[2 * i],
                   cpu_data[2 * i + 1], g[2 * i + 1], error);
        err_sum += error;
    }
    printf("Total Difference: %f \n", err_sum);
}

extern "C" void gpu_check_data(float *cpu_chi2, int nuv, float *visi, int data_size, float *mock_data, int image_size,
                               float *data_grad)
{
    if (!g_ctx) return;
    gpair_ctx *c = g_ctx;
    if (cpu_chi2 && gp_sync_scalars(c) == GPAIR_OK)
        printf("CPU chi2 %f GPU chi2 %f\n", *cpu_chi2, (float)c->sc_host->chi2);
    if (visi && c->have_problem && nuv <= c->nuv) {
        gpair_buf b = {(float *)c->visi, (size_t)2 * c->nuv, 100};
        gpu_compare_complex_data(nuv, visi, &b);
    }
    if (mock_data && c->have_problem && data_size <= c->ndata) {
        gpair_buf b = {c->mock, (size_t)c->ndata, 101};
        gpu_compare_data(data_size, mock_data, &b);
    }
    if (data_grad && image_size <= c->npix) gpu_compare_data(image_size, data_grad, &c->h_dg);
}
