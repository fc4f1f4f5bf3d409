/*
 * gpair_b200.h -- C ABI of the B200 (sm_100a) implementation of GPAIR's
 * image-reconstruction hot path.
 *
 * Two layers, both plain C (pointers and sizes only):
 *
 * 1. The reference's own GPU boundary, gpair1/trunk/gpu.h:5-120, with the same
 *    function names, argument order and meaning. OpenCL types are replaced by
 *    layout-identical structs (cl_float2 -> gpair_float2, cl_long4 ->
 *    gpair_long4, cl_short4 -> gpair_short4) and cl_mem* by the opaque
 *    gpair_buf*. As in the reference these functions use one global context,
 *    block until the device work is done, copy caller arrays in, and on error
 *    print a message and exit (print_opencl_error, gpair1/trunk/gpu.c:186-202)
 *    unless gpair_set_exit_on_error(0) was called.
 *
 * 2. Extensions: per-context handles, status codes instead of exit, device
 *    twiddle generation from (u, v), precision modes, a device-resident CG
 *    whose scalars never leave the GPU, and the host-side OIFITS indexer and
 *    setup routines the reference keeps in getoifits.c / gpair.c.
 *
 * Image layout everywhere: float[N*N], x fastest (index x + y*N), as in
 * gpair1/trunk/cpu.c:469. Data layout: data/data_err/mock are
 * [npow V2 values][nbis x (T3 real, T3 imaginary)] (gpair1/trunk/gpair.c:1003-1062).
 */
#ifndef GPAIR_B200_H
#define GPAIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define GPAIR_OK 0
#define GPAIR_ERR_INVALID (-1)   /* bad argument / size / state */
#define GPAIR_ERR_ALLOC (-2)     /* host or device allocation failed */
#define GPAIR_ERR_CUDA (-3)      /* a CUDA runtime call failed */
#define GPAIR_ERR_STATE (-4)     /* call out of order (e.g. no problem loaded) */
#define GPAIR_ERR_TIMEOUT (-5)   /* a bounded device wait gave up */
#define GPAIR_ERR_NO_DEVICE (-6) /* no CUDA device / not an sm_100 device */
#define GPAIR_ERR_NUMERIC (-7)   /* NaN or Inf reached a reduction */

/* ------------------------------------------------------------------ types */
typedef struct { float s0, s1; } gpair_float2;                /* cl_float2 */
typedef struct { int64_t s0, s1, s2, s3; } gpair_long4;       /* cl_long4 */
typedef struct { int16_t s0, s1, s2, s3; } gpair_short4;      /* cl_short4 */
typedef struct gpair_buf gpair_buf;                           /* cl_mem */
typedef struct gpair_ctx gpair_ctx;

/* oi_uv, gpair1/trunk/getoifits.h:53-59 */
typedef struct { float u, v, bandwidth, wavelength; } gpair_uv;

/* =========================================================================
 * Layer 1: the reference boundary (gpair1/trunk/gpu.h)
 * ========================================================================= */

/* gpu.h:5   -- print the message and code, release the GPU, exit(0) */
void print_opencl_error(char *error_message, int error_code);
/* gpu.h:7   -- human-readable name of a status code */
char *print_cl_errstring(int err);
/* gpu.h:9   -- copy data_size floats from buffer input to buffer output */
void gpu_backup_gradient(int data_size, gpair_buf *input, gpair_buf *output);
/* gpu.h:11  -- prepares device-side tables (twiddle operands, triangle map) */
void gpu_build_kernels(int data_size, int image_width, int image_size);
/* gpu.h:17  -- debug comparison of CPU results against the device's
 *             (prints like gpair1/trunk/gpu.c:501-612); NULL pointers are skipped */
void gpu_check_data(float *cpu_chi2, int nuv, float *visi /* complex64[nuv] */, int data_size,
                    float *mock_data, int image_size, float *data_grad);
/* gpu.h:22  */
void gpu_compare_data(int size, float *cpu_data, gpair_buf *pGpu_data);
/* gpu.h:24  */
void gpu_compare_complex_data(int size, float *cpu_data /* complex64 */, gpair_buf *pGpu_data);
/* gpu.h:26-28 -- gradient_buffer = data_gradient - alpha * entropy_gradient */
void gpu_compute_criterion_gradient(int image_width, float hyperparameter_entropy, gpair_buf *gradient_buffer);
void gpu_compute_criterion_gradient_curr(int image_width, float hyperparameter_entropy);
void gpu_compute_criterion_gradient_temp(int image_width, float hyperparameter_entropy);
/* gpu.h:30  -- temp_image = current_image + steplength * descent_direction (no clamp) */
void gpu_compute_criterion_step(int image_width, float steplength, float minvalue);
/* gpu.h:32-35 */
void gpu_compute_entropy(int image_width, gpair_buf *gpu_image, gpair_buf *entropy_storage);
void gpu_compute_entropy_gradient(int image_width, gpair_buf *gpu_image);
void gpu_compute_entropy_gradient_curr(int image_width);
void gpu_compute_entropy_gradient_temp(int image_width);
/* gpu.h:37  -- flux_storage = sum(image); flux_inverse_storage = 1/flux (on the device) */
void gpu_compute_flux(gpair_buf *gpu_image, gpair_buf *flux_storage, gpair_buf *flux_inverse_storage);
/* gpu.h:44-46 -- d chi2 / d image, from the visibilities and mock data of the
 *                immediately preceding gpu_get_chi2 on the same image */
void gpu_compute_data_gradient(gpair_buf *gpu_image, int nuv, int npow, int nbis, int image_width);
void gpu_compute_data_gradient_curr(int nuv, int npow, int nbis, int image_width);
void gpu_compute_data_gradient_temp(int nuv, int npow, int nbis, int image_width);
/* gpu.h:48  -- descent_direction = beta * descent_direction - full_gradient_new */
void gpu_compute_descent_dir(int image_width, float beta);
/* gpu.h:50  -- upload data (padded to data_size), biphasors, triangle references, prior */
void gpu_copy_data(float *data, float *data_err, int data_size, int data_size_uv, gpair_float2 *data_phasor,
                   int phasor_size, int pow_size, gpair_long4 *gpu_bsref_uvpnt, gpair_short4 *gpu_bsref_sign,
                   int bsref_size, float *default_model, int image_size, int image_width);
/* gpu.h:56  -- DFT tables in the transposed layout [x][uv] (i = nuv*x + uv), dft_size entries each */
void gpu_copy_dft(gpair_float2 *dft_x, gpair_float2 *dft_y, int dft_size);
/* gpu.h:58  -- upload the current image (x_size * y_size floats) */
void gpu_copy_image(float *image, int x_size, int y_size);
/* gpu.h:60  */
void gpu_cleanup(void);
/* gpu.h:62  -- chi2 of the current mock data (device-resident result) */
void gpu_data2chi2(int data_size);
/* gpu.h:64  */
int gpu_error_callback(char *error);
/* gpu.h:66-68 -- chi2 of the current / temporary / given image */
float gpu_get_chi2_curr(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv);
float gpu_get_chi2_temp(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv);
float gpu_get_chi2(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, gpair_buf *gpu_image);
/* gpu.h:70-72 -- Gull-Skilling entropy of the image */
float gpu_get_entropy(int image_width, gpair_buf *gpu_image);
float gpu_get_entropy_curr(int image_width);
float gpu_get_entropy_temp(int image_width);
/* gpu.h:74  -- blocking read of `size` floats of a device buffer into cpu_buffer */
float *gpu_get_image(int size, float *cpu_buffer, gpair_buf *gpu_image);
/* gpu.h:76  -- sum(array1 * array2) over data_width*data_height elements */
float gpu_get_scalprod(int data_width, int data_height, gpair_buf *array1, gpair_buf *array2);
/* gpu.h:78-84 -- borrowed handles of the device buffers */
gpair_buf *gpu_getp_ci(void);  /* current image */
gpair_buf *gpu_getp_ti(void);  /* temporary (trial) image */
gpair_buf *gpu_getp_fgn(void); /* full gradient, new */
gpair_buf *gpu_getp_fg(void);  /* full gradient, previous */
gpair_buf *gpu_getp_dd(void);  /* descent direction */
gpair_buf *gpu_getp_tg(void);  /* gradient at the trial image */
gpair_buf *gpu_getp_eg(void);  /* entropy gradient */
/* gpu.h:86-88 */
void gpu_image2chi2(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, gpair_buf *gpu_image);
void gpu_image2vis(int nuv, int data_alloc_uv, gpair_buf *gpu_image);
/* gpu.h:90  -- pick device 0 (or GPAIR_DEVICE), create the global context */
void gpu_init(void);
/* gpu.h:94  -- strong-Wolfe zoom between the two step lengths (gpair1/trunk/gpu.c:1947-2065) */
float gpu_linesearch_zoom(int nuv, int npow, int nbis, int data_alloc, int data_alloc_uv, int image_width,
                          float steplength_low, float steplength_high, float criterion_steplength_low,
                          float wolfe_product1, float criterion_init, int *criterion_evals, int *grad_evals,
                          gpair_buf *pDescent_direction, gpair_buf *pTemp_gradient, float hyperparameter_entropy);
/* The reference's zoom can loop forever once its bracket is two adjacent
 * floats; this one stops after a trial cap (200 by default) and returns
 * steplength_low. No counterpart in the reference: gpair_set_zoom_trial_cap
 * sets the cap (0 = 200), gpair_zoom_cap_hits counts the zoom calls that
 * stopped at it (each also writes gpair_last_error of the global context),
 * gpair_zoom_cap_hits_reset clears the count. */
int gpair_set_zoom_trial_cap(int cap);
int gpair_zoom_cap_hits(void);
void gpair_zoom_cap_hits_reset(void);
/* gpu.h:102 -- mock data + chi2 from the stored visibilities */
void gpu_new_chi2(int nuv, int npow, int nbis, int data_alloc);
/* gpu.h:104 -- V2 and T3 mock data from the stored visibilities */
void gpu_vis2data(gpair_buf *gpu_vis, int nuv, int npow, int nbis);
/* gpu.h:114 -- output = sum(array1 * array2) (device-resident) */
void gpu_scalar_prod(int data_width, int data_height, gpair_buf *array1, gpair_buf *array2, gpair_buf *output);
/* gpu.h:116 */
void gpu_shutdown(void);
/* gpu.h:118-119 -- image = max(image + steplength * d, minval); temp likewise into the temporary image */
void gpu_update_image(int image_width, float steplength, float minval, gpair_buf *descent_direction);
void gpu_update_tempimage(int image_width, float steplength, float minval, gpair_buf *descent_direction);

/* =========================================================================
 * Layer 2: extensions (status-returning, per-context)
 * ========================================================================= */

/* ---- host-side OIFITS indexing and setup (no device needed) ---- */

/* OI_WAVELENGTH / OI_VIS2 / OI_T3 tables (gpair1/trunk/exchange.h:63-141);
 * per-channel columns are row-major [numrec][nwave]. */
typedef struct {
    const char *insname;
    int nwave;
    const float *eff_wave, *eff_band;
} gpair_oi_wavelength;
typedef struct {
    const char *insname;
    long numrec;
    int nwave;
    const int *target_id;
    const double *vis2data, *vis2err, *ucoord, *vcoord;
    const char *flag;
} gpair_oi_vis2;
typedef struct {
    const char *insname;
    long numrec;
    int nwave;
    const int *target_id;
    const double *t3amp, *t3amperr, *t3phi, *t3phierr, *u1coord, *v1coord, *u2coord, *v2coord;
    const char *flag;
} gpair_oi_t3;

/* oi_data (gpair1/trunk/getoifits.h:61-75): arrays are malloc'd by
 * gpair_get_oi_fits_data and released by gpair_free_oi_data. */
typedef struct {
    int npow, nbis, nuv;
    float *pow, *powerr, *bisamp, *bisamperr, *bisphs, *bisphserr;
    gpair_uv *uv;     /* [nuv] */
    int64_t *uvpnt;   /* [nbis][3]: ab, bc, ca */
    int16_t *sign;    /* [nbis][3]: +1, or -1 when the uv point is conjugated */
} gpair_oi_data;

/* get_oi_fits_data, gpair1/trunk/getoifits.c:65-357 (bit-exact, hashed matcher). */
int gpair_get_oi_fits_data(int target_id, float minband, float maxband, int nwave_tables,
                           const gpair_oi_wavelength *waves, int nvis2_tables, const gpair_oi_vis2 *vis2,
                           int nt3_tables, const gpair_oi_t3 *t3, gpair_oi_data *out);
void gpair_free_oi_data(gpair_oi_data *d);

/* init_data, gpair1/trunk/gpair.c:997-1066. bisamp/bisamperr are updated in
 * place on extrapolation. data/data_err hold npow + 2*nbis floats, phasor nbis
 * complex values. Returns the change of ndof (<= 0). */
int gpair_init_data(int do_extrapolation, int npow, int nbis, const float *pow, const float *powerr,
                    float *bisamp, float *bisamperr, const float *bisphs, const float *bisphserr,
                    const int64_t *uvpnt, float *data, float *data_err, gpair_float2 *phasor);

/* set_model, gpair1/trunk/cpu.c:645-749 (types 0 flat, 1 Dirac, 2 disk, 3 Gaussian, 4 Lorentzian). */
int gpair_set_model(int image_width, float image_pixellation, int modeltype, float modelwidth, float modelflux,
                    float *default_model);

/* DFT tables, gpair1/trunk/gpair.c:231-245 (CPU layout [nuv][N]) and, when
 * dft_x_t/dft_y_t are non-NULL, the transposed device layout of
 * gpair1/trunk/gpair.c:615-627 ([N][nuv], zero-padded to dft_alloc entries). */
int gpair_dft_tables(int image_width, int nuv, const gpair_uv *uv, float pixellation, gpair_float2 *dft_x,
                     gpair_float2 *dft_y, gpair_float2 *dft_x_t, gpair_float2 *dft_y_t, int dft_alloc);

/* ---- device contexts ---- */

#define GPAIR_PREC_FP32 0     /* CUDA-core FP32 DFT/adjoint (FP32 twiddles) */
#define GPAIR_PREC_SPLIT16 1  /* tcgen05 f16 hi+lo split operands, 3 products, FP32 accumulate */
#define GPAIR_PREC_TF32 2     /* tcgen05 kind::tf32, TF32 operands, 1 product, FP32 accumulate */
#define GPAIR_PREC_TF32X3 3   /* tcgen05 kind::tf32, TF32 hi+lo split operands, 3 products, FP32 accumulate */
#define GPAIR_PREC_SPLIT16F8 4 /* forward: f16 hi*hi (kind::f16) plus the two hi*lo cross terms as E4M3
                                  products (kind::f8f6f4, twice the f16 rate) into the same FP32
                                  accumulator; adjoint: as GPAIR_PREC_SPLIT16 */

#define GPAIR_IMG_CURR 0
#define GPAIR_IMG_TEMP 1

int gpair_create(gpair_ctx **ctx, int device);
int gpair_destroy(gpair_ctx *ctx);
const char *gpair_strerror(int status);
/* 1 = reference behaviour (layer 1 prints and exits on error), 0 = return */
void gpair_set_exit_on_error(int on);
/* the context used by layer 1 (created by gpu_init) */
gpair_ctx *gpair_global_context(void);
/* last CUDA error string seen by a context */
const char *gpair_last_error(gpair_ctx *ctx);

/* Load a problem. uv: nuv points; data/data_err: npow + 2*nbis; phasor: nbis;
 * uvpnt/sign: [nbis][3]; default_model: N*N (copied). Twiddles are generated
 * on the device from uv in FP64 phase with argument reduction. */
int gpair_set_problem(gpair_ctx *ctx, int image_width, float pixellation, int nuv, const gpair_uv *uv, int npow,
                      int nbis, const float *data, const float *data_err, const gpair_float2 *phasor,
                      const int64_t *uvpnt, const int16_t *sign, const float *default_model);
int gpair_set_precision(gpair_ctx *ctx, int mode);
int gpair_get_precision(gpair_ctx *ctx);
int gpair_set_image(gpair_ctx *ctx, int which, const float *image);
int gpair_get_image(gpair_ctx *ctx, int which, float *image);

/* One criterion evaluation on the current or temporary image:
 * chi2 (FP64 sum), entropy S (FP64 sum); visibilities and mock data stay on the device. */
int gpair_criterion(gpair_ctx *ctx, int which, double *chi2, double *entropy);
/* Data gradient, entropy gradient and full gradient (data - alpha * entropy) of
 * the image last passed to gpair_criterion. The full gradient goes to the new
 * gradient (which = CURR) or the trial gradient (which = TEMP). */
int gpair_gradient(gpair_ctx *ctx, int which, float alpha);
/* read back device results of the last evaluation */
int gpair_get_visibilities(gpair_ctx *ctx, gpair_float2 *visi);      /* nuv */
int gpair_get_mock(gpair_ctx *ctx, float *mock);                     /* npow + 2*nbis */
int gpair_get_data_gradient(gpair_ctx *ctx, float *grad);            /* N*N */
int gpair_get_entropy_gradient(gpair_ctx *ctx, float *grad);         /* N*N */
int gpair_get_full_gradient(gpair_ctx *ctx, int which, float *grad); /* N*N */

/* Device-resident CG (reference control flow, FP64 scalars kept on the GPU). */
typedef struct {
    int method;       /* 0 SD, 1 FR, 2 PR+, 3 HS+ (the reference's beta rules, gpair.c:733-753);
                         4 projected L-BFGS (no reference counterpart): the newest 4 (s, y)
                         pairs in the compact form, pixels on the positivity bound with an
                         outward gradient held fixed; use wolfe2 = 0.9 with GPAIR_LS_WOLFE.
                         Not available in gpair_batch_run. A checkpoint does not hold the
                         pairs: a restored run rebuilds its history. */
    int iterations;
    float alpha;      /* entropy hyperparameter */
    double minvalue;  /* 1e-8 */
    double wolfe1;    /* 1e-4 */
    double wolfe2;    /* 0.1 */
    double step_max;  /* 100 */
    int max_zoom;     /* cap on zoom trials (reference: unbounded) */
    int max_bracket;  /* cap on bracketing trials */
    int resume;       /* 0: start a new run; 1: continue the previous run's CG state
                         (iteration count, previous gradient, descent direction) */
    int host_loop;    /* 0 (default): the whole run is one CUDA graph launch (conditional
                         nodes steer the line search on the device); 1: the host reads
                         the controller's decision after every trial */
    /* ---- extensions beyond the reference's CG ---- */
    int line_search;  /* GPAIR_LS_WOLFE (default): the reference's strong-Wolfe bracketing
                         and zoom, one trial image per evaluation. GPAIR_LS_BATCH: every
                         round evaluates GPAIR_LS_TRIALS trial images in one batched
                         evaluation (a geometric grid of steps around the last accepted
                         step, shifted until it brackets the best step, then one refine
                         round inside the bracket); the best trial is accepted */
    double target_J;  /* > 0: the run stops at the first iteration whose current image has
                         J <= target_J (time-to-objective runs); 0: off */
    double batch_step_max; /* GPAIR_LS_BATCH: largest trial step (default 1e12) */
    int *stop_flag;   /* device int shared by runs racing to target_J on one device (see
                         gpair_stop_flag_create), or NULL: the run that reaches target_J
                         first sets it; every run that sees it set ends at its next
                         iteration (a start-image race: a warm start against the flat
                         prior, each in its own context and stream) */
} gpair_cg_params;

#define GPAIR_LS_WOLFE 0
#define GPAIR_LS_BATCH 1
#define GPAIR_LS_TRIALS 8

typedef struct {
    int iterations_done;
    int criterion_evals;
    int grad_evals;
    double J, chi2, entropy; /* at the start of the last iteration */
    double last_step, last_beta;
    int status;
    int reached;  /* 1 when the run stopped at target_J */
    int stopped;  /* 1 when a racing run reached target_J first */
} gpair_cg_result;

/* Runs the same CG parameters on n contexts (one problem each, distinct contexts)
 * at once: every context's run is prepared, then every run's graph is launched on
 * its context's stream, then the host waits for all. Small problems that each fill
 * a few SMs run side by side this way (many independent reconstructions, e.g. a
 * survey or a training set). host_loop must be 0; res (length n) may be NULL.
 * Returns the first error; per-run status in res[i].status. */
int gpair_cg_run_many(gpair_ctx **ctx, int n, const gpair_cg_params *p, gpair_cg_result *res);

/* Regulariser S of the criterion J = chi2 - alpha S (default Gull-Skilling entropy,
 * gpair1/trunk/cpu.c:385-412). GPAIR_REG_L2: S = sum over m > 0 of -I^2/(2m), dS/dI =
 * -I/m (gpair1/trunk/cpu.c:508-521; the reference's L2_entropy_gradient returns only
 * the sum of this field). Applies to every evaluation and CG run of the context. */
#define GPAIR_REG_GULL_SKILLING 0
#define GPAIR_REG_L2 1
int gpair_set_regularizer(gpair_ctx *ctx, int kind);

/* Single-pixel update of the current image (the move of annealing / MCMC samplers;
 * the corrected form of gpair1/trunk/gpu.c:2137-2182 and gpair1/trunk/cpu.c:477-486):
 * pixel (x, y) becomes `value`, V_k <- (F V_k + delta e_k(x,y)) / (F + delta) in FP64,
 * then V2/T3, chi2 and S are recomputed from V in O(nuv + nbis) work, no DFT. Needs a
 * preceding gpair_criterion on the current image; a gpair_gradient may follow.
 * Returns the new chi2 and regulariser S (either pointer may be NULL). */
int gpair_update_pixel(gpair_ctx *ctx, int x, int y, float value, double *chi2, double *entropy);

/* Checkpoint / resume of a CG run: the device controller state (iteration, beta
 * history, line-search state), the image, the descent direction and the gradients,
 * as one host buffer of gpair_cg_checkpoint_size() bytes (a versioned header, then
 * raw data). After gpair_cg_checkpoint_load on a context holding the same problem,
 * gpair_cg_run with resume = 1 continues exactly where the saved run stopped. */
size_t gpair_cg_checkpoint_size(gpair_ctx *ctx);
int gpair_cg_checkpoint_save(gpair_ctx *ctx, void *buffer, size_t bytes);
int gpair_cg_checkpoint_load(gpair_ctx *ctx, const void *buffer, size_t bytes);

/* Batched reconstructions: one CUDA graph holds the whole CG loop of every context
 * (each an independent branch with its own conditional nodes), so one graph launch
 * runs all n reconstructions and the device schedules their kernels side by side.
 * Create after every context holds its problem, image, precision and (optional)
 * autotuned configuration; those are fixed into the graph: rebuild the batch after
 * changing any of them. gpair_batch_run takes the same parameters as gpair_cg_run
 * (line_search must match the batch's, host_loop must be 0; no traces) and returns
 * per-context results; each context's last_run_stats holds the batch's device time.
 *
 * Lockstep batches (the default of gpair_batch_create when line_search is
 * GPAIR_LS_BATCH and some context is on a tensor-core path): the reconstructions
 * advance one CG step at a time together.
 *   Staged (gpair_batch_grouped = 2; every context on a tensor-core path with one
 *   operand element type -- f16 or TF32 -- and given by (u, v), n <= 4096): every
 *   stage of an iteration (image prep, V2/T3/chi2, adjoint weights and operand,
 *   gradient, direction, trial prep, trial chi2, image update, controller) is ONE
 *   launch over all instances, and every contraction (criterion forward, adjoint,
 *   trial forward) one grouped tcgen05 launch per class of contexts with the same
 *   operand kind, product count and tile layout (at most 256 per launch), with
 *   per-instance operand maps and arguments in device memory.
 *   Forwards only (gpair_batch_grouped = 1; otherwise, or with
 *   GPAIR_BATCH_FORWARDS_ONLY): each instance runs its own stage kernels; the
 *   trial forwards of every tensor-core class are grouped launches.
 * Each instance's results are bitwise those of its separate run. Otherwise, or with
 * GPAIR_BATCH_INDEPENDENT, every context's loop is an independent graph branch
 * (gpair_batch_grouped = 0). gpair_batch_run returns GPAIR_ERR_STATE when a
 * context's operand or batch buffers were rebuilt since the batch was created
 * (another precision, tile layout, problem or image size). */
typedef struct gpair_batch gpair_batch;
#define GPAIR_BATCH_INDEPENDENT 1
#define GPAIR_BATCH_FORWARDS_ONLY 2
/* Staged batches only: a device timer stamp (ns) after every launch of an
 * iteration, for a breakdown of where an iteration's time goes. The stamps
 * themselves add one small kernel per launch. */
#define GPAIR_BATCH_STAGE_STAMPS 4
/* Staged batches only: passes of image rows per block of the grouped trial-image
 * prep, p = 1, 2, 4, ..., 32 (0 or absent: the smallest that brings the launch
 * within four waves of resident blocks). Trial images at most 256 pixels wide sum
 * their flux and regulariser per image row, so p changes no result; wider ones
 * keep the grid of their single launch. gpair_batch_prep_passes returns the
 * passes a staged batch uses (0: not staged). */
#define GPAIR_BATCH_PREP_PASSES(p) (((p) & 63) << 8)
int gpair_batch_create(gpair_batch **batch, gpair_ctx **ctx, int n, int line_search);
int gpair_batch_create_ex(gpair_batch **batch, gpair_ctx **ctx, int n, int line_search, int flags);
int gpair_batch_grouped(const gpair_batch *batch);
int gpair_batch_prep_passes(const gpair_batch *batch);
/* Stage stamps of a batch created with GPAIR_BATCH_STAGE_STAMPS; returns the
 * number of words (39), or 0 without stamps. Positions 0-18: the device timer
 * (ns) at the pre-phase start, then after the image prep, criterion forwards,
 * V2/T3/chi2, c_k, W, adjoints, gradient, direction and router; a batched
 * evaluation's start, then after the trial prep, trial forwards, trial chi2
 * and router; the post-phase start, then after the image update, controller
 * and router (the last values of the run). Words 19-37: the time since the
 * stamp before each position, summed over every iteration and batched
 * evaluation since the last reset (0 at the three starts). Word 38: batched
 * evaluations since the last reset. reset != 0 zeroes the words afterwards. */
int gpair_batch_stage_stamps(const gpair_batch *batch, unsigned long long *ns, int max, int reset);
int gpair_batch_run(gpair_batch *batch, const gpair_cg_params *p, gpair_cg_result *results);
int gpair_batch_destroy(gpair_batch *batch);

/* Stop flag for racing runs: a device int, zeroed at creation and by reset. */
int gpair_stop_flag_create(int **flag);
int gpair_stop_flag_reset(int *flag);
int gpair_stop_flag_destroy(int *flag);

/* Adjoint DFT of uv-plane weights: image[y*N + x] = Re sum_k w_k Fx[k][x] Fy[k][y]
 * (the dirty image of the weights). Overwrites the evaluation state of the
 * context (a gpair_gradient call must follow a new gpair_criterion). */
int gpair_adjoint_image(gpair_ctx *ctx, const gpair_float2 *weights, float *image);

/* ---- warm-start network kernels (no counterpart in the reference) ----
 * Building blocks of the learned warm start: a 3x3-convolution encoder/decoder
 * trained and run by the library's own kernels. Device pointers, float NCHW
 * activations, 3x3 weights [Cout][Cin][3][3] as bfloat16 (uint16 storage),
 * FP32 accumulation; `stream` is a cudaStream_t (NULL: the default stream).
 * Every call returns GPAIR_OK, GPAIR_ERR_INVALID (bad sizes) or GPAIR_ERR_CUDA. */
int gpair_cnn_conv3x3(const float *in, const void *w_bf16, const float *bias, const float *skip, float *out, int B,
                      int Cin, int Cout, int H, int W, int relu, void *stream);
int gpair_cnn_conv3x3_bwd_data(const float *gout, const void *w_bf16, float *gin, int B, int Cin, int Cout, int H,
                               int W, int accumulate, void *stream);
int gpair_cnn_conv3x3_bwd_weight(const float *in, const float *gpre, float *dw, float *db, float *scratch,
                                 long long scratch_floats, int B, int Cin, int Cout, int H, int W, void *stream);
int gpair_cnn_relu_mask(const float *y, float *g, long long n, void *stream);
int gpair_cnn_pool2(const float *in, float *out, long long BC, int H, int W, void *stream);
int gpair_cnn_pool2_bwd(const float *gout, float *gin, long long BC, int H, int W, int accumulate, void *stream);
int gpair_cnn_up2(const float *in, float *out, long long BC, int H, int W, void *stream);
int gpair_cnn_up2_bwd(const float *gout, float *gin, long long BC, int H, int W, void *stream);
int gpair_cnn_head(const float *d, const float *w, const float *bias, float *z, float *out, float *asum, int B, int C,
                   int HW, void *stream);
int gpair_cnn_head_bwd(const float *d, const float *w, const float *z, const float *out, const float *asum,
                       const float *gout, float *gd, float *dw, float *scratch, int B, int C, int HW, void *stream);
/* mode 0: loss_b = HW sum (out - t)^2; mode 1: loss_b = sum (out - t)^2 / sum t^2 */
int gpair_cnn_mse(const float *out, const float *target, float *gout, double *loss, int B, int HW, float gscale,
                  int mode, void *stream);
int gpair_cnn_adam(float *p, void *p_bf16, const float *g, float *m, float *v, int n, float lr, float b1, float b2,
                   float eps, int step, void *stream);
int gpair_cnn_to_bf16(const float *src, void *dst, int n, void *stream);

void gpair_cg_default_params(gpair_cg_params *p);
/* Runs p->iterations CG iterations from the current image. Per-iteration
 * trace arrays (length p->iterations) may be NULL. */
int gpair_cg_run(gpair_ctx *ctx, const gpair_cg_params *p, gpair_cg_result *res, double *trace_J,
                 double *trace_chi2, double *trace_entropy, double *trace_step, double *trace_beta);

/* Timing hooks for benchmarks: device time of the last gpair_cg_run (ms) and
 * the algorithmic DFT + adjoint flop count it executed. */
int gpair_last_run_stats(gpair_ctx *ctx, double *device_ms, double *dft_flops, int *kernel_launches);

/* Stages of one criterion + gradient evaluation, timed with CUDA events on
 * the context's stream (average ms over `reps` repetitions, on the current
 * image): [0] image prep (flux, entropy), [1] forward DFT, [2] V2/T3/chi2 and
 * adjoint weights, [3] per-uv weight gather, [4] adjoint DFT, [5] gradient
 * finalize. Returns the number of stages written (<= max_stages). */
#define GPAIR_NSTAGES 6
int gpair_time_stages(gpair_ctx *ctx, int reps, double *stage_ms, int max_stages);

/* The stages of one batched line-search evaluation (GPAIR_LS_TRIALS trial images),
 * timed like gpair_time_stages: [0] trial images + operands, [1] forward contraction
 * of the stack, [2] chi2 of every trial. Uses the steps of the last batch. */
int gpair_time_batch_stages(gpair_ctx *ctx, int reps, double *stage_ms, int max_stages);

/* Autotuner: times criterion + gradient evaluations of the loaded problem (current
 * image) under candidate configurations and keeps the fastest. Candidates: the
 * precision path (GPAIR_TUNE_PRECISION: FP32 CUDA cores, split-f16 or split-f16/E4M3
 * tensor cores; all meet the 1e-5 accuracy bounds on the benchmark workloads, though
 * split-f16/E4M3's chi2 error can pass 1e-5 where |V| is far below the total flux at
 * most uv points, as for a pixel-by-pixel random image), the adjoint's split-K tile length
 * (GPAIR_TUNE_SPLITS: half, default and double the heuristic's K-blocks per split,
 * within the FP32-accumulation cap) and the tensor-core tile (GPAIR_TUNE_TILE:
 * 256 x 256 output tiles on CTA pairs or 128 x 256 on single CTAs, as
 * gpair_set_tc_pair selects). GPAIR_TUNE_CACHE reuses the choice made for a
 * problem of the same device, width and uv count (to 1/8) and objective in this
 * process, made with the same precision path and tile when those are not tuned. */
#define GPAIR_TUNE_PRECISION 1
#define GPAIR_TUNE_SPLITS 2
#define GPAIR_TUNE_CACHE 4
#define GPAIR_TUNE_BATCHED 8 /* objective: criterion + gradient + 2 batched 8-trial evaluations
                                (one batched-line-search iteration) instead of criterion + gradient */
#define GPAIR_TUNE_TILE 16
#define GPAIR_TUNE_MAX_CANDIDATES 16
typedef struct {
    int precision;       /* chosen precision mode */
    int adjoint_splits;  /* chosen split-K count of the adjoint contraction */
    double ms_per_eval;  /* criterion + gradient, chosen configuration */
    int from_cache;
    int n_candidates;
    int tile_m;          /* chosen tensor-core tile rows: 256 (CTA pairs), 128, or 0 (CUDA cores) */
    int cand_precision[GPAIR_TUNE_MAX_CANDIDATES];
    int cand_splits[GPAIR_TUNE_MAX_CANDIDATES];
    int cand_tile_m[GPAIR_TUNE_MAX_CANDIDATES];
    double cand_ms[GPAIR_TUNE_MAX_CANDIDATES];
} gpair_tune_result;
int gpair_autotune(gpair_ctx *ctx, int flags, int reps, gpair_tune_result *result);

/* Live stage timing inside gpair_cg_run: when on, every stage launch of the
 * run is bracketed by CUDA events on the context's stream;
 * gpair_last_run_stage_ms returns the summed ms and launch count per stage
 * (same stage order as gpair_time_stages) of the last run. */
int gpair_set_stage_timing(gpair_ctx *ctx, int on);

/* ---- failure path of the tensor-core kernels ----
 * No counterpart in the reference, which prints and exits on any device error
 * (gpair1/trunk/gpu.c:186-202). Every pipeline wait of the tcgen05 kernels is
 * bounded by a clock budget (default about 2 s: budget_cycles = 0); when one
 * runs out the kernel stops its roles, waits for its TMA copies in flight,
 * frees its tensor memory and returns, and the call reports GPAIR_ERR_TIMEOUT
 * with the context still usable. skip_loads = 1 is a test switch: the TMA
 * producer issues no loads, so the MMA and epilogue waits run out with no
 * copy in flight. (0, 0) restores the defaults. */
int gpair_set_tc_wait(gpair_ctx *ctx, long long budget_cycles, int skip_loads);

/* ---- tensor-core contraction layout ----
 * No counterpart in the reference. on = 1 (default): the forward DFT and the
 * adjoint run on pairs of CTAs (a cluster of two SMs sharing one 256 x 256
 * tcgen05.mma.cta_group::2 tile, each SM staging half of the image-side
 * operand, 3 pipeline stages); on = 0: one CTA per 128 x 256 tile, 2 stages.
 * Results agree to rounding; the operands are rebuilt on a change. */
int gpair_set_tc_pair(gpair_ctx *ctx, int on);
int gpair_get_tc_pair(gpair_ctx *ctx);

/* ---- overlapped kernel launches ----
 * No counterpart in the reference. on = 1 (default; environment variable
 * GPAIR_PDL=0 makes 0 the default of new contexts): the kernels of an
 * evaluation are launched as programmatic dependent launches, so that each
 * kernel's launch and block scheduling overlap the end of the kernel before it
 * (each waits for that kernel's completion before it touches memory). Results
 * are the same either way; captured graphs are rebuilt on a change. */
int gpair_set_pdl(gpair_ctx *ctx, int on);

/* ---- split-K lengths for contexts that share the GPU ----
 * No counterpart in the reference. The adjoint contraction of a context alone
 * splits its K dimension (2 nuv) so that its units fill every SM, which for a
 * small image means many short splits and many partial images to write and sum.
 * For n contexts run together (gpair_cg_run_many, gpair_batch_*), this sets each
 * tensor-core context's split-K length so that all their units together fill
 * the SMs about twice, each context's share in proportion to its adjoint work
 * (at most the FP32-accumulation cap per split), and the gradient's sum of the
 * partial images to one thread per four pixels (a context alone spreads a small
 * image's sum over up to 8). The split-K lengths of CUDA-core contexts are left
 * as they are. Results change by rounding only; call before capturing a batch. */
int gpair_set_shared_splits(gpair_ctx **ctx, int n);
int gpair_last_run_stage_ms(gpair_ctx *ctx, double *stage_ms, int *stage_launches, int max_stages);

/* ---- allocation-free data stage ----
 * No counterpart in the reference. For callers that cannot allocate device
 * memory: programs whose own allocator owns the device heap, and latency-
 * critical loops where a cudaMalloc could serialise the device. It computes
 * the V2 / T3 mock data and chi2 (FP64 sum) from visibilities, like
 * gpu_vis2data + gpu_data2chi2. It allocates nothing: every pointer is a
 * caller-owned DEVICE buffer in the reference's layouts (visi float2[nuv],
 * data/data_err/mock float[npow + 2*nbis], phasor float2[nbis], uvpnt
 * long4[nbis], sign short4[nbis], chi2 one double). The reduction scratch is
 * a fixed 64 KiB device array inside the library, held by every GPU that
 * loads it until the process exits. Limits: npow + nbis <= 2,097,152,
 * npow <= nuv; larger sizes return GPAIR_ERR_INVALID without launching.
 * The first call on a device looks up the scratch address for that device
 * (with it current); make that first call before any stream capture. The call
 * is asynchronous on `stream` (a cudaStream_t of the current device, NULL =
 * default stream; a stream of another device returns GPAIR_ERR_INVALID);
 * results are valid once the stream has reached it. All calls share the one scratch
 * array, so calls that overlap on the GPU (other streams, other host threads)
 * race and must be serialised by the caller. An out-of-range triangle
 * reference is not read; the call then writes chi2 = NaN. */
int gpair_vis2data_chi2_noalloc(const gpair_float2 *visi, int nuv, int npow, int nbis, const float *data,
                                const float *data_err, const gpair_float2 *phasor, const gpair_long4 *uvpnt,
                                const gpair_short4 *sign, float *mock, double *chi2, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GPAIR_B200_H */
