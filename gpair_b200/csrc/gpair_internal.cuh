// gpair_internal.cuh -- device context, HBM layout and shared helpers of the
// B200 reconstruction path. Not part of the public ABI.
//
// HBM layout of one problem (N = image width, K = nuv, T = nbis):
//   images        image, image_temp, model, grads: float[N*N], x fastest
//   data          data, data_err, mock: float[npow + 2T]
//   triangles     tri: int4 {ab, bc, ca, sign bits} (bit j set = vertex j conjugated)
//                 phasor: float2[T]
//   uv            uvc: float2[K] (u, v in wavelengths)
//   twiddles      fx, fy: float2[K][N]  (Fx[k][x] = e^{+2 pi i s u_k x}, Fy[k][y] = e^{-2 pi i s v_k y})
//                 generated on the device with FP64 phase and argument reduction
//   forward       vpart: float2[MT][K], per-row-tile partial visibilities (before 1/F)
//                 visd: double2[K] (1/F included), visi: float2[K] (the reference's visi)
//   adjoint       trib: float2[T][3] per-vertex adjoint weights, inc_off/inc_idx: CSR map
//                 uv -> incident (triangle, vertex); cw: float2[K] summed weights c_k
//                 gpart: float[S][N*N] split-K partial adjoint images
//   scalars       DevScalars (FP64 sums, CG state) + reduction partials
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "gpair_b200.h"

#define GP_THREADS 256
#define GP_MAX_PARTIALS 4096
#define GP_MAX_STAGE_REC 8192

// Reduction slots (index into DevScalars::counter / partial areas)
enum {
    RED_PREP = 0,  // flux, entropy
    RED_CHI2 = 1,  // chi2
    RED_ADJ = 2,   // C = Re sum c_k V_k, max |c_k|
    RED_GRAD = 3,  // gradient finalize dots
    RED_DIR = 4,   // descent direction dot
    RED_DOT = 5,   // generic scalar product
    RED_LBP = 6,   // projected L-BFGS: candidate pair dots
    RED_LBD = 7,   // projected L-BFGS: dots of the projected gradient
    RED_NSLOTS = 8
};

// CG line-search actions decided on the device
enum { CG_EVAL_CRIT = 1, CG_EVAL_GRAD = 2, CG_DONE = 3, CG_EVAL_BATCH = 4 };
enum { CG_PH_BRACKET = 0, CG_PH_ZOOM = 1 };

// batched line search (GPAIR_LS_BATCH)
#define GP_NTR GPAIR_LS_TRIALS  // trial images per batched evaluation
#define GP_LS_RATIO 4.0         // step ratio of the geometric grid
#define GP_LS_RATIO_LOG2 2      // log2 of GP_LS_RATIO: grid steps are exact power-of-two multiples
#define GP_LS_MAX_ROUNDS 6      // grid shifts + refine per iteration
#define GP_LS_MAX_PTS (GP_LS_MAX_ROUNDS * GP_NTR)
enum { BR_GRID = 0, BR_REFINE = 1 };

// projected L-BFGS direction (method 4): pairs kept, and the dot products the
// pair kernel (3 of the candidate, 2 per stored pair) and the direction-dots
// kernel (q.q, 2 per stored pair) reduce
#define GP_LB_PAIRS 4
#define GP_LB_NPD (3 + 2 * GP_LB_PAIRS)
#define GP_LB_NQD (1 + 2 * GP_LB_PAIRS)

struct CgState {
    // parameters
    int method, max_zoom, max_bracket;
    int run_limit;  // iterations this run performs (graph-captured runs)
    double alpha, minvalue, c1, c2, step_max;
    int ls_mode;            // GPAIR_LS_WOLFE / GPAIR_LS_BATCH
    double target_J;        // stop once the current image has J <= target_J (0: off)
    double batch_step_max;  // largest batched trial step
    // per iteration
    int it;
    double J, chi2, entropy, beta, wolfe1;
    double prev_nn;  // g_new.g_new of the previous iteration (= g_old.g_old now)
    // bracketing
    int phase, ls_it, action, zoom_counter, zoom_trials, bracket_trials;
    double s, s_old, J_init, J_old, Jt;
    // zoom
    double lo, hi, J_lo, z_s, z_s_old, z_J_old;
    double sel;
    // counters
    int criterion_evals, grad_evals;
    int run_it;  // iterations completed in this run
    int batches;  // batched trial evaluations in this run
    int reached;  // target objective reached
    int stopped;  // a racing run reached the target first
    // batched line search
    int bphase, bround, npts, force_sd;
    double s_c;
    double ts[GP_NTR];                 // steps of the batch being evaluated
    double pts_s[GP_LS_MAX_PTS], pts_J[GP_LS_MAX_PTS];  // points evaluated this iteration
    // projected L-BFGS (method 4): logical pairs 0 (oldest) .. lb_count - 1
    // live in the buffers lb_slot[0 .. lb_count - 1] of the GP_LB_PAIRS + 1
    // image-sized S and Y buffers; lb_slot[GP_LB_PAIRS] is the free buffer the
    // next candidate pair is written to
    int lb_count, lb_xvalid, lb_drop;
    int lb_slot[GP_LB_PAIRS + 1];
    double lb_sy[GP_LB_PAIRS][GP_LB_PAIRS];  // s_i . y_j (upper triangle used)
    double lb_yy[GP_LB_PAIRS][GP_LB_PAIRS];  // y_i . y_j
    double lb_gamma;                          // H0 = gamma I, from the newest accepted pair
    // direction d = -(lb_cq q + sum_i lb_cs[i] s_i + sum_i lb_cy[i] y_i), q = projected gradient
    double lb_cq, lb_cs[GP_LB_PAIRS], lb_cy[GP_LB_PAIRS];
};

struct DevScalars {
    double flux, invflux, entropy, chi2;
    double imax;          // max |image| of the last prepared image
    double adj_c;      // C = Re sum_k c_k V_k
    double cmax;       // max |c_k| (scaling of split operands)
    double gscale;     // factor applied to the summed adjoint partials (1, or 1/operand scales)
    double grad_dots[2][4];  // [CURR/TEMP]: g.g, g.g_old, g.d, d.g_old
    double dir_dot;    // d.g_new after the descent update
    double dot;        // generic scalar product
    float flux_f, invflux_f, chi2_f, entropy_f, dot_f;
    unsigned int counter[RED_NSLOTS];
    unsigned int nonfinite;  // set when a NaN/Inf reaches a reduction
    unsigned int tc_err;     // tensor-core kernels: bounded wait gave up (bit = which wait)
    // batched trials: per-trial flux, entropy and chi2
    double t_flux[GP_NTR], t_invflux[GP_NTR], t_entropy[GP_NTR], t_chi2[GP_NTR];
    unsigned int t_counter[GP_NTR + 1];
    int *stop_flag;  // shared with racing runs (device memory), or null
    int reg_kind;    // GPAIR_REG_GULL_SKILLING / GPAIR_REG_L2
    // single-pixel update: old total flux and flux change of the last update
    double upd_flux_old, upd_delta;
    // projected L-BFGS reductions
    double lb_pdots[GP_LB_NPD], lb_qdots[GP_LB_NQD];
    CgState cg;
};

// Regulariser term of one pixel and its gradient.
//   Gull-Skilling (gpair1/trunk/cpu.c:385-412): I - m - I ln(I/m), or -m where I <= 0
//   or m <= 0; gradient -ln(I/m), the previous value kept where I <= 0 or m <= 0.
//   L2 (gpair1/trunk/cpu.c:508-521): -I^2 / (2m) where m > 0, else 0; gradient -I/m
//   where m > 0, else 0 (the reference's L2_entropy_gradient returns only the sum
//   of this field).
__device__ __forceinline__ double reg_term(double I, double m, int kind)
{
    if (kind == GPAIR_REG_L2) return m > 0.0 ? -I * I / (2.0 * m) : 0.0;
    return (I > 0.0 && m > 0.0) ? (I - m - I * log(I / m)) : -m;
}
// The same term in FP32 without cancellation, for sums accumulated in FP64.
// With r = (I - m) / m: I - m - I ln(I/m) = m g(r),
//   g(r) = r - (1 + r) ln(1 + r) = -r^2 sum_{k>=0} (-r)^k / ((k + 1)(k + 2)),
// evaluated by the series (Horner, k <= 18: truncation below 2^-26 of the sum)
// for |r| < 1/2, where I - m is exact (Sterbenz); elsewhere the closed form
// (I - m) - I ln(I/m), whose two terms cancel by at most a factor of 6.
// Relative error of a term: a few units of 2^-24.
__device__ __forceinline__ float reg_term_f(float I, float m, int kind)
{
    if (kind == GPAIR_REG_L2) return m > 0.f ? -I * I / (2.f * m) : 0.f;
    if (!(I > 0.f && m > 0.f)) return -m;
    const float dlt = I - m;
    if (fabsf(dlt) < 0.5f * m) {
        const float r = dlt / m, t = -r;
        float p = 1.f / 380.f;  // k = 18: 1 / (19 * 20)
#pragma unroll
        for (int k = 17; k >= 0; k--) p = fmaf(p, t, 1.f / (float)((k + 1) * (k + 2)));
        return m * (-(r * r) * p);
    }
    return dlt - I * logf(I / m);
}
// reg_term_f of eight pixels, summed into `acc` in pixel order: the series is
// evaluated for all eight at once (independent FMA chains, no branch), the
// closed form only for pixels far from the prior. Same values as reg_term_f.
__device__ __forceinline__ void reg_terms8(const float (&I)[8], const float (&m)[8], int kind, double &acc)
{
    float term[8];
    if (kind == GPAIR_REG_L2) {
#pragma unroll
        for (int k = 0; k < 8; k++) term[k] = m[k] > 0.f ? -I[k] * I[k] / (2.f * m[k]) : 0.f;
    } else {
        float r[8], p[8];
        bool near[8];
        bool any_far = false;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const float dlt = I[k] - m[k];
            near[k] = I[k] > 0.f && m[k] > 0.f && fabsf(dlt) < 0.5f * m[k];
            any_far |= !near[k];
            r[k] = near[k] ? dlt / m[k] : 0.f;
            p[k] = 1.f / 380.f;
        }
#pragma unroll
        for (int j = 17; j >= 0; j--) {
            const float cj = 1.f / (float)((j + 1) * (j + 2));
#pragma unroll
            for (int k = 0; k < 8; k++) p[k] = fmaf(p[k], -r[k], cj);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) term[k] = m[k] * (-(r[k] * r[k]) * p[k]);
        if (any_far) {
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (!near[k]) term[k] = (I[k] > 0.f && m[k] > 0.f) ? (I[k] - m[k]) - I[k] * logf(I[k] / m[k]) : -m[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 8; k++) acc += (double)term[k];
}

// A graph-captured CG run goes on after an iteration (the end-of-iteration
// test of the controller)
__device__ __forceinline__ bool cg_run_goes_on(const DevScalars *sc)
{
    const CgState &s = sc->cg;
    return s.run_it < s.run_limit && !sc->nonfinite && !sc->tc_err && !s.reached && !s.stopped;
}

__device__ __forceinline__ float reg_grad(float I, float m, float prev, int kind)
{
    if (kind == GPAIR_REG_L2) return m > 0.f ? (float)(-(double)I / (double)m) : 0.f;
    return (I > 0.f && m > 0.f) ? (float)(-log((double)I / (double)m)) : prev;
}

struct gpair_buf {
    float *ptr;
    size_t count;  // floats
    int id;
};

struct gpair_ctx {
    int device;
    cudaStream_t stream;
    char last_error[256];
    int precision;

    // problem
    int N, npix, nuv, npow, nbis, ndata;
    float pix;
    int have_problem, have_image;
    int have_uv;      // the problem came with (u, v) (else: the reference's DFT tables only)
    int mt;           // number of row tiles of the forward DFT
    int splits;       // split-K factor of the last adjoint (number of partial images)
    int splits_simt;  // split-K factor of the CUDA-core adjoint
    int gpart_cap;    // partial images gpart holds

    // buffers
    float *image, *image_temp, *model;
    float *data, *data_err, *mock;
    int4 *tri;
    float2 *phasor;
    float2 *uvc;
    float2 *fx, *fy;
    float2 *vpart;
    double2 *visd;
    float2 *visi;
    float2 *trib, *cw;
    int *inc_off, *inc_idx;
    float *gpart;
    float *data_grad, *entropy_grad, *full_grad_new, *full_grad, *grad_temp, *descent_dir;
    double *partials;  // RED_NSLOTS * GP_MAX_PARTIALS * 4 doubles
    DevScalars *sc;
    DevScalars *sc_host;  // pinned mirror for reads

    // tensor-core operand buffers (GPAIR_PREC_SPLIT16 / TF32), see umma path
    void *tc_state;

    // handles for layer 1
    gpair_buf h_image, h_image_temp, h_fgn, h_fg, h_dd, h_tg, h_eg, h_dg, h_model;

    // timing / stats of the last gpair_cg_run
    double last_ms, last_flops;
    long long launches;       // running count of kernel launches
    long long last_launches;  // launches of the last gpair_cg_run
    int last_image_src;  // which image the last criterion used (0/1), -1 none

    // live stage timing inside gpair_cg_run (events on the context stream)
    int stage_timing;
    cudaEvent_t *st_ev;   // 2 * GP_MAX_STAGE_REC events
    int *st_stage;        // stage id per record
    int st_n;
    double stage_ms[8];
    int stage_cnt[8];

    // batched line-search trials: GP_NTR trial images, partial visibilities
    // vpart_b[GP_NTR * epp][K] (epp row-tile entries per trial), reduction partials
    float *image_trials;
    // projected L-BFGS (method 4): GP_LB_PAIRS + 1 image-sized buffers each of
    // steps s and gradient changes y, and the image the last direction started from
    float *lb_s, *lb_y, *lb_xold;
    float2 *vpart_b;
    double2 *visb;  // visibilities of the GP_NTR trials [GP_NTR][K], when their partial entries are many
    double *partials_b;
    int batch_wave[2];  // blocks per trial that fill one wave: [0] trial prep, [1] trial chi2
    int epp;  // forward partial entries per trial image

    // graph-captured CG (cg_graph.cu): one graph per line-search mode, so that
    // alternating modes does not re-capture; cg_graph_mode = the mode last run
    void *cg_graph[2];
    int cg_graph_mode;
    int cg_method;  // direction method of the current run (4: projected L-BFGS passes in the graph)
    // controller fused into the next reduction kernel launched (-1: none)
    int fuse_ctrl, fuse_handles;
    unsigned long long fh_iter, fh_ls, fh_grad;

    // reference-boundary staging (layer 1)
    gpair_float2 *ref_dft_x, *ref_dft_y;  // host copies of the transposed tables
    int ref_dft_size;
    float *ref_data, *ref_data_err, *ref_model;
    gpair_float2 *ref_phasor;
    gpair_long4 *ref_uvpnt;
    gpair_short4 *ref_sign;
    int ref_data_size, ref_phasor_size, ref_bsref_size, ref_npow;
    int bound_nuv, bound_npow, bound_nbis;

    // tensor-core kernels: clock budget of each pipeline wait (0 = default)
    // and a failure-path test switch: the TMA producer issues no loads, so
    // the MMA and epilogue waits run out with no copy in flight
    long long tc_wait_budget;
    int tc_skip_loads;
    // lockstep batches: device flag gating this context's batched-trial kernels (or null)
    const int *gate;
    // bumped whenever the tensor operands or the batch buffers are freed: graphs
    // captured before hold stale pointers
    unsigned int buf_gen;
    // tensor-core contractions on CTA pairs (tcgen05 cta_group::2) instead of single CTAs
    int tc_pair;
    // programmatic dependent launches of the evaluation chain (gp_launch), default on
    int pdl;
    // most threads per four pixels in the gradient's split sum (k_grad_finalize): 8 alone,
    // 1 for contexts that share the GPU (gpair_set_shared_splits)
    int gf_parts;
};

// ---------------------------------------------------------------- helpers
#define GP_CUDA(ctx, call)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            snprintf((ctx)->last_error, sizeof((ctx)->last_error), "%s: %s (%s:%d)", #call,        \
                     cudaGetErrorString(e_), __FILE__, __LINE__);                                   \
            return GPAIR_ERR_CUDA;                                                                  \
        }                                                                                           \
    } while (0)

#define GP_LAUNCH_CHECK(ctx)                                                                        \
    do {                                                                                            \
        (ctx)->launches++;                                                                          \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess) {                                                                    \
            snprintf((ctx)->last_error, sizeof((ctx)->last_error), "launch: %s (%s:%d)",           \
                     cudaGetErrorString(e_), __FILE__, __LINE__);                                   \
            return GPAIR_ERR_CUDA;                                                                  \
        }                                                                                           \
    } while (0)

static inline int gp_cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// a launch through gp_launch / gp_launch_on (its own error return), then the usual check
#define GP_LAUNCH(ctx, call)                                                                        \
    do {                                                                                            \
        cudaError_t le_ = (call);                                                                   \
        if (le_ != cudaSuccess) {                                                                   \
            snprintf((ctx)->last_error, sizeof((ctx)->last_error), "launch: %s (%s:%d)",           \
                     cudaGetErrorString(le_), __FILE__, __LINE__);                                  \
            return GPAIR_ERR_CUDA;                                                                  \
        }                                                                                           \
        GP_LAUNCH_CHECK(ctx);                                                                       \
    } while (0)

// ------------------------------------------ programmatic dependent launches
//
// The kernels of the evaluation chain are launched with programmatic stream
// serialization (gp_launch, when c->pdl is set): the next kernel on the stream
// is launched as the current one finishes, so that its launch overlaps the
// current kernel's last blocks instead of following its completion. Every
// kernel launched this way waits (gp_pdl_wait: griddepcontrol.wait, the full
// completion and memory flush of the kernel before it) before it reads or
// writes global memory. No kernel signals its dependents early
// (griddepcontrol.launch_dependents): dependent blocks made resident at a
// kernel's start and left waiting slowed the 256^2 evaluation chain by 7 %
// (measured), so the dependents launch as the blocks of the kernel before them
// exit. Launched without the attribute, the wait is a no-op.
__device__ __forceinline__ void gp_pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void gp_pdl_enter() { gp_pdl_wait(); }

template <typename... KP, typename... A>
static inline cudaError_t gp_launch_on(cudaStream_t st, int pdl, void (*k)(KP...), dim3 grid, dim3 block,
                                       size_t smem, A &&...args)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, static_cast<A &&>(args)...);
}

template <typename... KP, typename... A>
static inline cudaError_t gp_launch(gpair_ctx *c, void (*k)(KP...), dim3 grid, dim3 block, size_t smem, A &&...args)
{
    return gp_launch_on(c->stream, c->pdl, k, grid, block, smem, static_cast<A &&>(args)...);
}

// stage timing (context.cu): bracket the launches of one stage
void gp_stage_begin(gpair_ctx *c, int stage);
void gp_stage_end(gpair_ctx *c);

// kernel launchers (kernels_core.cu)
int gp_gen_twiddles(gpair_ctx *c);
int gp_twiddles_from_ref_tables(gpair_ctx *c, const float2 *dft_x_t, const float2 *dft_y_t);
int gp_build_incidence(gpair_ctx *c, const int64_t *uvpnt);
int gp_prep_image(gpair_ctx *c, int which, int trial_mode, double step_host, int step_from_state);
int gp_forward(gpair_ctx *c, int which);
int gp_vis_data(gpair_ctx *c);
int gp_adjoint(gpair_ctx *c, int which);
int gp_adj_weights_only(gpair_ctx *c);
int gp_adjoint_contraction(gpair_ctx *c, int which);
int gp_grad_finalize(gpair_ctx *c, int which, int mode, float alpha);
int gp_entropy_gradient(gpair_ctx *c, int which);
int gp_criterion_gradient(gpair_ctx *c, float alpha, float *out);
int gp_dot(gpair_ctx *c, const float *a, const float *b, int n);
int gp_descent_dir(gpair_ctx *c, int beta_from_state, double beta_host);
int gp_update_image(gpair_ctx *c, int step_from_state, double step_host, double minval, int backup);
int gp_update_temp(gpair_ctx *c, double step, double minval, int clamp);
int gp_cg_kernel(gpair_ctx *c, int which_ctrl);
// graph-captured controller: also sets the conditional handles of the CG graph
int gp_cg_kernel_graph(gpair_ctx *c, int which_ctrl, unsigned long long h_iter, unsigned long long h_ls,
                       unsigned long long h_grad, double *trace, int trace_cap);
int gp_sync_scalars(gpair_ctx *c);

enum { GRAD_FUSED = 0, GRAD_DATA_ONLY = 1 };
enum { CTRL_BEGIN = 0, CTRL_AFTER_DIR = 1, CTRL_AFTER_CRIT = 2, CTRL_AFTER_GRAD = 3, CTRL_INIT = 4, CTRL_RESUME = 5,
       CTRL_END = 6, CTRL_AFTER_BATCH = 7, CTRL_LB_PAIR = 8, CTRL_LB_COEF = 9 };

// batched line-search trials (kernels_core.cu / umma_dft.cu)
int gp_adjoint_image(gpair_ctx *c, const float2 *cw_host, float *out_host);
int gp_update_pixel(gpair_ctx *c, int x, int y, float value);
int gp_batch_alloc(gpair_ctx *c);
int gp_eval_batch_part(gpair_ctx *c, int part);
void gp_batch_free(gpair_ctx *c);
int gp_eval_batch(gpair_ctx *c);
int gp_eval_batch_timed(gpair_ctx *c, cudaEvent_t *ev);
int gp_tc_batch_prepare(gpair_ctx *c, int *epp);
int gp_trials_prep_launch(gpair_ctx *c);
int gp_tc_trials_prep_split(gpair_ctx *c, double *partials);
int gp_tc_forward_batch_gemm(gpair_ctx *c);

// tensor-core path (umma_dft.cu); return GPAIR_ERR_STATE when unavailable
int gp_tc_prepare(gpair_ctx *c);
int gp_tc_forward(gpair_ctx *c, int which);
int gp_tc_forward_gemm(gpair_ctx *c);
int gp_tc_split(gpair_ctx *c, int which);
int gp_tc_prep_image(gpair_ctx *c, int which);
// grouped contractions over several instances (lockstep batches): the forward of
// the batched trials (GP_TCG_TRIALS), the forward of the current image
// (GP_TCG_IMAGE) or the adjoint into split-K partial images (GP_TCG_ADJOINT)
enum { GP_TCG_TRIALS = 0, GP_TCG_IMAGE = 1, GP_TCG_ADJOINT = 2 };
int gp_tc_group_key(gpair_ctx *c);
int gp_tc_group_build(gpair_ctx **ctx, int n, const int *gate, unsigned int *err, void **out);
int gp_tc_group_build_kind(gpair_ctx **ctx, int n, int kind, const int *gate, unsigned int *err, void **out);
int gp_tc_group_forward(void *grp, gpair_ctx *c);
int gp_tc_group_run(void *grp, gpair_ctx *c, cudaStream_t st);
void gp_tc_group_free(void *grp);
// forward row tiles and adjoint split count of a context's tensor state (what
// its forward and adjoint launches would set in c->mt and c->splits)
int gp_tc_stage_sizes(gpair_ctx *c, int *mt, int *splits);
int gp_tc_forward_entries(int N);
int gp_tc_shared_splits(gpair_ctx **ctx, int n);

// Grouped stage kernels (group.cuh): the argument struct of one instance for
// stage GS_* (host memory, gp_stage_args_size bytes) and its virtual grid's
// block count; one launch over n instances whose argument structs are at
// d_args (device) with block starts d_start[0..n], gated by gate[i].
// GS_CTRL_END writes its trace row to `trace` (capacity 1).
enum {
    GS_PREP_IMAGE = 0,   // current image: flux, regulariser, max, forward operand (umma_dft.cu)
    GS_VIS_DATA = 1,     // V, V2/T3, chi2, adjoint weights (no controller)
    GS_ADJ_WEIGHTS = 2,  // c_k and C
    GS_BUILD_W = 3,      // adjoint weight operand (umma_dft.cu)
    GS_GRAD_FINALIZE = 4,  // gradient of the current image, then CTRL_BEGIN
    GS_DESCENT = 5,      // CG direction, then CTRL_AFTER_DIR
    GS_PREP_TRIALS = 6,  // batched trial images and their operands (umma_dft.cu)
    GS_CHI2_BATCH = 7,   // chi2 of every trial, then CTRL_AFTER_BATCH
    GS_UPDATE = 8,       // image update with the accepted step, gradient backup
    GS_CTRL_END = 9,     // end of the iteration (trace row)
    GS_COUNT = 10
};
size_t gp_stage_args_size(int stage);
int gp_stage_args(gpair_ctx *c, int stage, double *trace, void *out, int *nblocks);
int gp_stage_group_launch(gpair_ctx *c, int stage, const void *d_args, const int *d_start, int n, int total,
                          const int *gate);
// the umma_dft.cu stages (GS_PREP_IMAGE, GS_PREP_TRIALS, GS_BUILD_W); `op` is the
// operand kind of every instance in the launch
size_t gp_tc_stage_args_size(int stage);
// passes: GS_PREP_TRIALS only, passes of rows per block (1: the single launch's grid)
int gp_tc_stage_args(gpair_ctx *c, int stage, void *out, int *nblocks, int *op, int passes = 1);
int gp_tc_prep_trials_passes(gpair_ctx *const *ctx, int n, int op);
int gp_tc_stage_group_launch(gpair_ctx *c, int stage, int op, const void *d_args, const int *d_start, int n,
                             int total, const int *gate);
int gp_tc_build_w(gpair_ctx *c);
int gp_tc_adjoint_gemm(gpair_ctx *c);
int gp_tc_prep_split_trial(gpair_ctx *c);
int gp_tc_splits(int N, int nuv, int nsm, int bk, int pair, int *kb_per_out);
int gp_lbfgs_alloc(gpair_ctx *c);
void gp_lbfgs_free(gpair_ctx *c);
int gp_lbfgs_direction(gpair_ctx *c);
int gp_tc_max_splits(int N, int nuv, int nsm);
int gp_tc_kb_cap(gpair_ctx *c);
int gp_tc_adjoint(gpair_ctx *c, int which);
void gp_tc_free(gpair_ctx *c);
int gp_tc_kb_per(gpair_ctx *c);
int gp_tc_set_kb_per(gpair_ctx *c, int kb_per);
int gp_tc_split_count(gpair_ctx *c, int kb_per);
int gp_eval_criterion(gpair_ctx *c, int which, int trial);
int gp_eval_gradient(gpair_ctx *c, int which, float alpha);
void gp_cg_graph_free(gpair_ctx *c);
