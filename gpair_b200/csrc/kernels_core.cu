// kernels_core.cu -- device kernels of the reconstruction path (everything
// except the tcgen05 contractions, which live in umma_dft.cu).
//
//   k_gen_twiddles   Fx, Fy tables from (u, v), FP64 phase in turns reduced to
//                    [-1/2, 1/2] before sincospi (the reference builds them on the
//                    host in double, gpair1/trunk/gpair.c:231-245)
//   k_prep           image (or trial image max(I + s d, minval)) -> flux and
//                    Gull-Skilling entropy, FP64 sums (gpu.c:860-884, cpu.c:385-400,
//                    kernel_update_tempimage.cl)
//   k_fwd_simt       forward DFT on CUDA cores: T = I Fx^T per row tile, reduced
//                    against Fy in the epilogue (kernel_visi.cl / cpu.c:449-475)
//   k_vis_data       V = sum of row-tile partials / F; V2, T3, chi2 (FP64 sum) and
//                    the adjoint weights of every V2 point and triangle vertex
//                    (kernel_pow_spec.cl, kernel_bispec.cl, kernel_chi2.cl,
//                    cpu.c:758-802, cpu.c:371-383)
//   k_adj_weights    c_k = a_k + sum of incident triangle-vertex weights (CSR
//                    gather, fixed order), C = Re sum c_k V_k
//   k_adj_simt       adjoint image G[y][x] = Re sum_k c_k Fy[k][y] Fx[k][x],
//                    split over k (kernel_grad_pow.cl + kernel_grad_bis.cl, cpu.c:279-369)
//   k_grad_finalize  data grad = sum of splits - C; entropy gradient (previous
//                    value kept where I <= 0 or m <= 0); full gradient and the CG
//                    dot products in FP64 (kernel_entropy_gs_grad.cl,
//                    kernel_criterion_grad.cl)
//   k_descent, k_update_image, k_update_temp, k_dot, k_cg_ctrl
//                    CG vectors and the line-search state machine of
//                    gpair1/trunk/gpair.c:682-915 and gpair1/trunk/gpu.c:1947-2065,
//                    with FP64 scalars that stay on the device.
#include <cuda_fp16.h>
#include <math.h>
#include <string.h>

#include "gpair_internal.cuh"

#define RPMAS_D ((3.14159265358979323 / 180.0) / 3600000.0)

#include "group.cuh"
#include "reduce.cuh"
#include "umma.cuh"

__device__ void cg_control(DevScalars *__restrict__ sc, int what);
__device__ void cg_set_handles(DevScalars *__restrict__ sc, int what, cudaGraphConditionalHandle h_iter,
                               cudaGraphConditionalHandle h_ls, cudaGraphConditionalHandle h_grad);

// Controller fused into the last block of a reduction kernel (thread 0 only)
struct FusedCtrl {
    int what;         // CTRL_* to run after the reduction, or -1
    int use_handles;  // set the CG graph's conditionals (graph-captured runs only)
    cudaGraphConditionalHandle h_iter, h_ls, h_grad;
};

__device__ __forceinline__ void run_fused_ctrl(DevScalars *sc, const FusedCtrl &f)
{
    if (f.what < 0) return;
    cg_control(sc, f.what);
    if (f.use_handles) cg_set_handles(sc, f.what, f.h_iter, f.h_ls, f.h_grad);
}

static FusedCtrl take_fused_ctrl(gpair_ctx *c)
{
    FusedCtrl f;
    f.what = c->fuse_ctrl;
    f.use_handles = c->fuse_handles;
    f.h_iter = c->fh_iter;
    f.h_ls = c->fh_ls;
    f.h_grad = c->fh_grad;
    c->fuse_ctrl = -1;
    return f;
}

static inline double *slot_partials(gpair_ctx *c, int slot) { return c->partials + (size_t)slot * GP_MAX_PARTIALS * 4; }

// ------------------------------------------------------------- twiddles

__global__ void k_gen_twiddles(const float2 *__restrict__ uvc, int nuv, int N, float pix, float2 *__restrict__ fx,
                               float2 *__restrict__ fy)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nuv * N) return;
    int k = (int)(idx / N), i = (int)(idx % N);
    float2 uv = uvc[k];
    // phase / (2 pi) in turns, FP64, then reduced to [-1/2, 1/2]
    double tu = RPMAS_D * (double)pix * (double)uv.x * (double)i;
    double tv = RPMAS_D * (double)pix * (double)uv.y * (double)i;
    tu -= rint(tu);
    tv -= rint(tv);
    double su, cu, sv, cv;
    sincospi(2.0 * tu, &su, &cu);
    sincospi(2.0 * tv, &sv, &cv);
    fx[idx] = make_float2((float)cu, (float)su);   // e^{+2 pi i s u x}
    fy[idx] = make_float2((float)cv, (float)(-sv)); // e^{-2 pi i s v y}
}

int gp_gen_twiddles(gpair_ctx *c)
{
    long long n = (long long)c->nuv * c->N;
    if (n == 0) return GPAIR_OK;
    k_gen_twiddles<<<gp_cdiv(n, 256), 256, 0, c->stream>>>(c->uvc, c->nuv, c->N, c->pix, c->fx, c->fy);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// transposed reference tables [x][uv] -> [uv][x]
__global__ void k_transpose_tables(const float2 *__restrict__ tx, const float2 *__restrict__ ty, int nuv, int N,
                                   float2 *__restrict__ fx, float2 *__restrict__ fy)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nuv * N) return;
    int k = (int)(idx / N), i = (int)(idx % N);
    fx[idx] = tx[(size_t)nuv * i + k];
    fy[idx] = ty[(size_t)nuv * i + k];
}

int gp_twiddles_from_ref_tables(gpair_ctx *c, const float2 *dft_x_t, const float2 *dft_y_t)
{
    size_t n = (size_t)c->nuv * c->N;
    if (n == 0) return GPAIR_OK;
    float2 *tx = nullptr, *ty = nullptr;
    GP_CUDA(c, cudaMallocAsync(&tx, n * sizeof(float2), c->stream));
    GP_CUDA(c, cudaMallocAsync(&ty, n * sizeof(float2), c->stream));
    GP_CUDA(c, cudaMemcpyAsync(tx, dft_x_t, n * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    GP_CUDA(c, cudaMemcpyAsync(ty, dft_y_t, n * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    k_transpose_tables<<<gp_cdiv((long long)n, 256), 256, 0, c->stream>>>(tx, ty, c->nuv, c->N, c->fx, c->fy);
    GP_LAUNCH_CHECK(c);
    GP_CUDA(c, cudaFreeAsync(tx, c->stream));
    GP_CUDA(c, cudaFreeAsync(ty, c->stream));
    return GPAIR_OK;
}

// ---------------------------------------------------------- image prep

// src: image to evaluate. In trial mode the evaluated image is
// max(src + s d, minval), written to dst. Sums flux and entropy in FP64.
__global__ void __launch_bounds__(GP_THREADS) k_prep(const float *__restrict__ src, const float *__restrict__ d,
                                                     float *__restrict__ dst, const float *__restrict__ model,
                                                     int npix, int trial, double step, int step_from_state,
                                                     double minval, double *__restrict__ partials,
                                                     DevScalars *__restrict__ sc)
{
    __shared__ double smem[2 * 32];
    double s = step_from_state ? sc->cg.s : step;
    if (step_from_state) minval = sc->cg.minvalue;
    double acc[2] = {0.0, 0.0};
    double mx = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float I = src[p];
        if (trial) {
            double t = (double)I + s * (double)d[p];
            if (t < minval) t = minval;
            I = (float)t;
            dst[p] = I;
        }
        double Id = I, m = model[p];
        acc[0] += Id;
        acc[1] += reg_term(Id, m, sc->reg_kind);
        mx = fmax(mx, fabs(Id));
    }
    block_sum<2>(acc, smem);
    mx = block_max(mx, smem);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x] = acc[0];
        partials[3 * blockIdx.x + 1] = acc[1];
        partials[3 * blockIdx.x + 2] = mx;
    }
    if (last_block(&sc->counter[RED_PREP])) {
        double v[2] = {0.0, 0.0}, m = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
            v[0] += __ldcg(&partials[3 * b]);
            v[1] += __ldcg(&partials[3 * b + 1]);
            m = fmax(m, __ldcg(&partials[3 * b + 2]));
        }
        block_sum<2>(v, smem);
        m = block_max(m, smem);
        if (threadIdx.x == 0) {
            sc->flux = v[0];
            sc->invflux = 1.0 / v[0];
            sc->entropy = v[1];
            sc->imax = m;
            sc->flux_f = (float)v[0];
            sc->invflux_f = (float)(1.0 / v[0]);
            sc->entropy_f = (float)v[1];
            if (!isfinite(v[0]) || !isfinite(v[1])) sc->nonfinite |= 1u;
            sc->counter[RED_PREP] = 0;
        }
    }
}

static int red_grid(long long n) { int g = gp_cdiv(n, GP_THREADS * 4); return g < 1 ? 1 : (g > 1184 ? 1184 : g); }

int gp_prep_image(gpair_ctx *c, int which, int trial_mode, double step_host, int step_from_state)
{
    const float *src = (which == GPAIR_IMG_TEMP && !trial_mode) ? c->image_temp : c->image;
    const int g = red_grid(c->npix);  // one wave, several pixels per thread: a short reduction tail
    k_prep<<<g, GP_THREADS, 0, c->stream>>>(src, c->descent_dir, c->image_temp, c->model, c->npix, trial_mode,
                                            step_host, step_from_state, (double)1e-8, slot_partials(c, RED_PREP),
                                            c->sc);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// ----------------------------------------------------- forward, CUDA cores

#define FB_M 64
#define FB_K 32
#define FB_X 32

__global__ void __launch_bounds__(256) k_fwd_simt(const float *__restrict__ img, const float2 *__restrict__ fx,
                                                  const float2 *__restrict__ fy, int N, int nuv,
                                                  float2 *__restrict__ vpart, const int *__restrict__ gate)
{
    if (gate && !*gate) return;  // lockstep batches: this instance's line search is over
    __shared__ float As[FB_X][FB_M + 1];
    __shared__ float2 Bs[FB_X][FB_K + 1];
    __shared__ float2 red[16][FB_K + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int k0 = blockIdx.x * FB_K, y0 = blockIdx.y * FB_M;
    // batched trials: image z of a stack, partials of image z after those of images < z
    img += (size_t)blockIdx.z * N * N;
    vpart += (size_t)blockIdx.z * gridDim.y * nuv;
    float2 acc[4][2];
#pragma unroll
    for (int r = 0; r < 4; r++) acc[r][0] = acc[r][1] = make_float2(0.f, 0.f);
    for (int x0 = 0; x0 < N; x0 += FB_X) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            int r = (tid >> 5) + 8 * i, cx = tid & 31, y = y0 + r, x = x0 + cx;
            As[cx][r] = (y < N && x < N) ? img[(size_t)y * N + x] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int kk = (tid >> 5) + 8 * i, cx = tid & 31, k = k0 + kk, x = x0 + cx;
            Bs[cx][kk] = (k < nuv && x < N) ? fx[(size_t)k * N + x] : make_float2(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll 8
        for (int cx = 0; cx < FB_X; cx++) {
            float2 b0 = Bs[cx][tx * 2], b1 = Bs[cx][tx * 2 + 1];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                float a = As[cx][ty * 4 + r];
                acc[r][0].x = fmaf(a, b0.x, acc[r][0].x);
                acc[r][0].y = fmaf(a, b0.y, acc[r][0].y);
                acc[r][1].x = fmaf(a, b1.x, acc[r][1].x);
                acc[r][1].y = fmaf(a, b1.y, acc[r][1].y);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        int k = k0 + tx * 2 + j;
        float2 part = make_float2(0.f, 0.f);
        if (k < nuv) {
#pragma unroll
            for (int r = 0; r < 4; r++) {
                int y = y0 + ty * 4 + r;
                if (y < N) {
                    float2 f = fy[(size_t)k * N + y];
                    part.x += acc[r][j].x * f.x - acc[r][j].y * f.y;
                    part.y += acc[r][j].x * f.y + acc[r][j].y * f.x;
                }
            }
        }
        red[ty][tx * 2 + j] = part;
    }
    __syncthreads();
    if (tid < FB_K) {
        float2 s = make_float2(0.f, 0.f);
        for (int r = 0; r < 16; r++) { s.x += red[r][tid].x; s.y += red[r][tid].y; }
        int k = k0 + tid;
        if (k < nuv) vpart[(size_t)blockIdx.y * nuv + k] = s;
    }
}

int gp_forward(gpair_ctx *c, int which)
{
    if (c->precision != GPAIR_PREC_FP32) {
        int rc = gp_tc_forward(c, which);
        if (rc != GPAIR_ERR_STATE) return rc;
        return GPAIR_ERR_STATE; // tensor path requested but unavailable: fail loudly
    }
    const float *img = (which == GPAIR_IMG_TEMP) ? c->image_temp : c->image;
    c->mt = gp_cdiv(c->N, FB_M);
    dim3 grid(gp_cdiv(c->nuv, FB_K), c->mt);
    k_fwd_simt<<<grid, 256, 0, c->stream>>>(img, c->fx, c->fy, c->N, c->nuv, c->vpart, nullptr);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// ------------------------------------------------- V2, T3, chi2, weights

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ double2 sum_vpart(const float2 *__restrict__ vpart, int mt, int nuv, int k, double invF)
{
    double re = 0.0, im = 0.0;
    for (int m = 0; m < mt; m++) {
        float2 p = vpart[(size_t)m * nuv + k];
        re += p.x;
        im += p.y;
    }
    return make_double2(re * invF, im * invF);
}

struct VisDataArgs {
    const float2 *vpart;
    int mt, nuv, npow, nbis;
    const float *data, *data_err;
    const int4 *tri;
    const float2 *phasor;
    int nblk_uv;
    double2 *visd;
    float2 *visi;
    float *mock;
    float2 *cw, *trib;
    double *partials;
    DevScalars *sc;
    FusedCtrl fc;
    int direct;
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void vis_data_body(const VisDataArgs &A, const GpVGrid &vg)
{
    const float2 *__restrict__ vpart = A.vpart;
    const int mt = A.mt, nuv = A.nuv, npow = A.npow, nbis = A.nbis, nblk_uv = A.nblk_uv, direct = A.direct;
    const float *__restrict__ data = A.data;
    const float *__restrict__ data_err = A.data_err;
    const int4 *__restrict__ tri = A.tri;
    const float2 *__restrict__ phasor = A.phasor;
    double2 *__restrict__ visd = A.visd;
    float2 *__restrict__ visi = A.visi;
    float *__restrict__ mock = A.mock;
    float2 *__restrict__ cw = A.cw;
    float2 *__restrict__ trib = A.trib;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    // direct: the visibilities are already in visd (a single-pixel update), not in vpart
    __shared__ double smem[32];
    const double invF = sc->invflux;
#define VIS_AT(k) (direct ? visd[(k)] : sum_vpart(vpart, mt, nuv, (k), invF))
    double chi[1] = {0.0};
    if (vg.bx < nblk_uv) {
        for (int k = vg.bx * blockDim.x + threadIdx.x; k < nuv; k += nblk_uv * blockDim.x) {
            double2 V = VIS_AT(k);
            visd[k] = V;
            visi[k] = make_float2((float)V.x, (float)V.y);
            float2 a = make_float2(0.f, 0.f);
            if (k < npow) {
                double m2 = V.x * V.x + V.y * V.y;
                mock[k] = (float)m2;
                double w = data_err[k], res = m2 - (double)data[k], r = res * w;
                chi[0] += r * r;
                double f = 4.0 * w * w * res * invF; // a_k = f conj(V_k)
                a = make_float2((float)(f * V.x), (float)(-f * V.y));
            }
            cw[k] = a;
        }
    } else {
        const int nblk_tri = vg.nbx - nblk_uv;
        for (int t = (vg.bx - nblk_uv) * blockDim.x + threadIdx.x; t < nbis; t += nblk_tri * blockDim.x) {
            int4 q = tri[t];
            double2 va = VIS_AT(q.x);
            double2 vb = VIS_AT(q.y);
            double2 vc = VIS_AT(q.z);
            if (q.w & 1) va = cconj(va);
            if (q.w & 2) vb = cconj(vb);
            if (q.w & 4) vc = cconj(vc);
            float2 phf = phasor[t];
            double2 ph = make_double2(phf.x, phf.y);
            double2 t3 = cmul(cmul(cmul(va, vb), vc), ph);
            int r0 = npow + 2 * t;
            mock[r0] = (float)t3.x;
            mock[r0 + 1] = (float)t3.y;
            double wre = data_err[r0], wim = data_err[r0 + 1];
            double rre = t3.x - (double)data[r0], rim = t3.y - (double)data[r0 + 1];
            chi[0] += (rre * wre) * (rre * wre) + (rim * wim) * (rim * wim);
            // adjoint: Re(conj(g) * t3der) with g = 2 w_re^2 (T3re - d_re) + i 2 w_im^2 T3im
            // (the reference uses the mock imaginary part alone, gpair1/trunk/cpu.c:364-365)
            double2 g = make_double2(2.0 * wre * wre * rre, 2.0 * wim * wim * t3.y);
            double2 base = cmul(cconj(g), ph);
            base.x *= invF;
            base.y *= invF;
            double2 bab = cmul(base, cmul(vb, vc));
            double2 bbc = cmul(base, cmul(va, vc));
            double2 bca = cmul(base, cmul(va, vb));
            if (q.w & 1) bab = cconj(bab);
            if (q.w & 2) bbc = cconj(bbc);
            if (q.w & 4) bca = cconj(bca);
            trib[3 * (size_t)t + 0] = make_float2((float)bab.x, (float)bab.y);
            trib[3 * (size_t)t + 1] = make_float2((float)bbc.x, (float)bbc.y);
            trib[3 * (size_t)t + 2] = make_float2((float)bca.x, (float)bca.y);
        }
    }
    block_sum<1>(chi, smem);
    if (threadIdx.x == 0) partials[vg.bx] = chi[0];
    if (last_block_of(&sc->counter[RED_CHI2], vg.nbx)) {
        double out[1];
        finish_sum<1>(partials, vg.nbx, out, smem);
        if (threadIdx.x == 0) {
            sc->chi2 = out[0];
            sc->chi2_f = (float)out[0];
            if (!isfinite(out[0])) sc->nonfinite |= 2u;
            sc->counter[RED_CHI2] = 0;
            run_fused_ctrl(sc, A.fc);
        }
    }
}

#undef VIS_AT

__global__ void __launch_bounds__(GP_THREADS) k_vis_data(const VisDataArgs a)
{
    gp_pdl_enter();
    vis_data_body(a, gp_vgrid_hw());
}

struct VisDataOp {
    using Args = VisDataArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { vis_data_body(a, v); }
};

static VisDataArgs vis_data_args(gpair_ctx *c, int direct, FusedCtrl fc)
{
    int nbu = gp_cdiv(c->nuv, GP_THREADS);
    if (nbu > 512) nbu = 512;
    if (nbu < 1) nbu = 1;
    int nbt = gp_cdiv(c->nbis, GP_THREADS);
    if (nbt > 1536) nbt = 1536;
    VisDataArgs a = {c->vpart, c->mt, c->nuv, c->npow, c->nbis, c->data, c->data_err, c->tri, c->phasor, nbu,
                     c->visd, c->visi, c->mock, c->cw, c->trib, slot_partials(c, RED_CHI2), c->sc, fc, direct,
                     nbu + nbt, 1};
    return a;
}

static int vis_data_launch(gpair_ctx *c, int direct);

int gp_vis_data(gpair_ctx *c) { return vis_data_launch(c, 0); }

// V_k = (sum of the forward's partial entries, in entry order) / F into visd: with
// many entries per uv point, summed once here instead of once per triangle vertex
// that gathers V_k (the same sum, so the same values)
__global__ void __launch_bounds__(GP_THREADS) k_vis_sum(const float2 *__restrict__ vpart, int mt, int nuv,
                                                        const DevScalars *__restrict__ sc,
                                                        double2 *__restrict__ visd)
{
    gp_pdl_enter();
    const double invF = sc->invflux;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nuv; k += gridDim.x * blockDim.x)
        visd[k] = sum_vpart(vpart, mt, nuv, k, invF);
}

// more partial entries than this: V is summed once (k_vis_sum) before the triangles gather it
#define VIS_PRESUM_ENTRIES 2

static int vis_data_launch(gpair_ctx *c, int direct)
{
    if (!direct && c->mt > VIS_PRESUM_ENTRIES && c->nuv > 0) {
        int nb = gp_cdiv(c->nuv, GP_THREADS);
        if (nb > 4 * 148) nb = 4 * 148;
        GP_LAUNCH(c, gp_launch(c, k_vis_sum, dim3(nb), dim3(GP_THREADS), 0, (const float2 *)c->vpart, c->mt, c->nuv,
                               (const DevScalars *)c->sc, c->visd));
        direct = 1;
    }
    const VisDataArgs a = vis_data_args(c, direct, take_fused_ctrl(c));
    GP_LAUNCH(c, gp_launch(c, k_vis_data, dim3(a.nbx), dim3(GP_THREADS), 0, a));
    return GPAIR_OK;
}

// ----------------------------------------------------- adjoint weights

struct AdjWeightsArgs {
    int nuv;
    const int *inc_off, *inc_idx;
    const float2 *trib;
    const double2 *visd;
    float2 *cw;
    double *partials;
    DevScalars *sc;
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void adj_weights_body(const AdjWeightsArgs &A, const GpVGrid &vg)
{
    const int nuv = A.nuv;
    const int *__restrict__ inc_off = A.inc_off;
    const int *__restrict__ inc_idx = A.inc_idx;
    const float2 *__restrict__ trib = A.trib;
    const double2 *__restrict__ visd = A.visd;
    float2 *__restrict__ cw = A.cw;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ double smem[32];
    double acc[1] = {0.0};
    double cmax = 0.0;
    for (int k = vg.bx * blockDim.x + threadIdx.x; k < nuv; k += vg.nbx * blockDim.x) {
        float2 a = cw[k];
        double re = a.x, im = a.y;
        const int pe = inc_off[k + 1];
        for (int p0 = inc_off[k]; p0 < pe; p0 += 8) {
            // up to 8 independent index loads, then 8 independent weight loads;
            // the sum keeps the ascending incidence order
            int idx[8];
#pragma unroll
            for (int j = 0; j < 8; j++) idx[j] = (p0 + j < pe) ? __ldg(&inc_idx[p0 + j]) : -1;
            float2 b[8];
#pragma unroll
            for (int j = 0; j < 8; j++) b[j] = idx[j] >= 0 ? __ldg(&trib[idx[j]]) : make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                re += b[j].x;
                im += b[j].y;
            }
        }
        float2 cf = make_float2((float)re, (float)im);
        cw[k] = cf;
        double2 V = visd[k];
        acc[0] += (double)cf.x * V.x - (double)cf.y * V.y;
        cmax = fmax(cmax, fmax(fabs((double)cf.x), fabs((double)cf.y)));
    }
    block_sum<1>(acc, smem);
    cmax = block_max(cmax, smem);
    if (threadIdx.x == 0) {
        partials[2 * vg.bx] = acc[0];
        partials[2 * vg.bx + 1] = cmax;
    }
    if (last_block_of(&sc->counter[RED_ADJ], vg.nbx)) {
        double s = 0.0, m = 0.0;
        for (int b = threadIdx.x; b < vg.nbx; b += blockDim.x) {
            s += __ldcg(&partials[2 * b]);
            m = fmax(m, __ldcg(&partials[2 * b + 1]));
        }
        double sv[1] = {s};
        block_sum<1>(sv, smem);
        m = block_max(m, smem);
        if (threadIdx.x == 0) {
            sc->adj_c = sv[0];
            sc->cmax = m;
            sc->gscale = 1.0;  // the tensor path's operand builder overrides this
            sc->counter[RED_ADJ] = 0;
        }
    }
}

__global__ void __launch_bounds__(GP_THREADS) k_adj_weights(const AdjWeightsArgs a)
{
    gp_pdl_enter();
    adj_weights_body(a, gp_vgrid_hw());
}

struct AdjWeightsOp {
    using Args = AdjWeightsArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { adj_weights_body(a, v); }
};

static AdjWeightsArgs adj_weights_args(gpair_ctx *c)
{
    int nb = gp_cdiv(c->nuv, GP_THREADS);
    if (nb > 592) nb = 592;
    if (nb < 1) nb = 1;
    AdjWeightsArgs a = {c->nuv, c->inc_off, c->inc_idx, c->trib, c->visd, c->cw, slot_partials(c, RED_ADJ), c->sc,
                        nb, 1};
    return a;
}

// ----------------------------------------------------- adjoint, CUDA cores

#define AB_M 64
#define AB_N 64
#define AB_K 16  // complex uv per k-step

__global__ void __launch_bounds__(256) k_adj_simt(const float2 *__restrict__ fx, const float2 *__restrict__ fy,
                                                  const float2 *__restrict__ cw, int N, int nuv, int kchunk,
                                                  float *__restrict__ gpart)
{
    __shared__ float As[2 * AB_K][AB_M + 4];
    __shared__ float Bs[2 * AB_K][AB_N + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int x0 = blockIdx.x * AB_N, y0 = blockIdx.y * AB_M;
    const int kb = blockIdx.z * kchunk, ke = min(nuv, kb + kchunk);
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int k0 = kb; k0 < ke; k0 += AB_K) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int kk = (tid >> 6) + 4 * i, cc = tid & 63, k = k0 + kk;
            float2 wa = make_float2(0.f, 0.f), fb = make_float2(0.f, 0.f);
            if (k < ke) {
                int y = y0 + cc, x = x0 + cc;
                float2 cwk = cw[k];
                if (y < N) {
                    float2 f = fy[(size_t)k * N + y];
                    wa = make_float2(cwk.x * f.x - cwk.y * f.y, cwk.x * f.y + cwk.y * f.x);
                }
                if (x < N) fb = fx[(size_t)k * N + x];
            }
            As[2 * kk][cc] = wa.x;
            As[2 * kk + 1][cc] = -wa.y;
            Bs[2 * kk][cc] = fb.x;
            Bs[2 * kk + 1][cc] = fb.y;
        }
        __syncthreads();
#pragma unroll 8
        for (int kp = 0; kp < 2 * AB_K; kp++) {
            float4 a = *reinterpret_cast<const float4 *>(&As[kp][ty * 4]);
            float4 b = *reinterpret_cast<const float4 *>(&Bs[kp][tx * 4]);
            float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    float *out = gpart + (size_t)blockIdx.z * N * N;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int y = y0 + ty * 4 + i;
        if (y >= N) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int x = x0 + tx * 4 + j;
            if (x < N) out[(size_t)y * N + x] = acc[i][j];
        }
    }
}

static int adj_splits(int N, int nuv)
{
    int tiles = gp_cdiv(N, AB_M) * gp_cdiv(N, AB_N);
    int s = gp_cdiv(148 * 3, tiles);
    int maxs = gp_cdiv(nuv, 64);
    if (s > maxs) s = maxs;
    if (s > 64) s = 64;
    return s < 1 ? 1 : s;
}

int gp_adj_weights_only(gpair_ctx *c)
{
    const AdjWeightsArgs a = adj_weights_args(c);
    GP_LAUNCH(c, gp_launch(c, k_adj_weights, dim3(a.nbx), dim3(GP_THREADS), 0, a));
    return GPAIR_OK;
}

// Adjoint of caller-given uv weights (already in cw): C = 0, max |c_k| for the
// tensor path's operand scale, unit adjoint scale.
__global__ void __launch_bounds__(GP_THREADS) k_adj_given(int nuv, const float2 *__restrict__ cw,
                                                          double *__restrict__ partials, DevScalars *__restrict__ sc)
{
    __shared__ double smem[32];
    double cmax = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nuv; k += gridDim.x * blockDim.x) {
        const float2 cf = cw[k];
        cmax = fmax(cmax, fmax(fabs((double)cf.x), fabs((double)cf.y)));
    }
    cmax = block_max(cmax, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = cmax;
    if (last_block(&sc->counter[RED_ADJ])) {
        double m = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) m = fmax(m, __ldcg(&partials[b]));
        m = block_max(m, smem);
        if (threadIdx.x == 0) {
            sc->adj_c = 0.0;
            sc->cmax = m;
            sc->gscale = 1.0;
            sc->counter[RED_ADJ] = 0;
        }
    }
}

int gp_adjoint_image(gpair_ctx *c, const float2 *cw_host, float *out_host)
{
    GP_CUDA(c, cudaMemcpyAsync(c->cw, cw_host, sizeof(float2) * c->nuv, cudaMemcpyHostToDevice, c->stream));
    int nb = gp_cdiv(c->nuv, GP_THREADS);
    if (nb > 592) nb = 592;
    if (nb < 1) nb = 1;
    k_adj_given<<<nb, GP_THREADS, 0, c->stream>>>(c->nuv, c->cw, slot_partials(c, RED_ADJ), c->sc);
    GP_LAUNCH_CHECK(c);
    int rc = gp_adjoint_contraction(c, GPAIR_IMG_CURR);
    if (rc) return rc;
    if ((rc = gp_grad_finalize(c, GPAIR_IMG_CURR, GRAD_DATA_ONLY, 0.f))) return rc;
    GP_CUDA(c, cudaMemcpyAsync(out_host, c->data_grad, sizeof(float) * c->npix, cudaMemcpyDeviceToHost, c->stream));
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

int gp_adjoint(gpair_ctx *c, int which)
{
    int rc = gp_adj_weights_only(c);
    if (rc) return rc;
    return gp_adjoint_contraction(c, which);
}

int gp_adjoint_contraction(gpair_ctx *c, int which)
{
    if (c->precision != GPAIR_PREC_FP32) return gp_tc_adjoint(c, which);
    int S = c->splits_simt;
    int kchunk = gp_cdiv(c->nuv, S);
    kchunk = gp_cdiv(kchunk, AB_K) * AB_K;
    S = gp_cdiv(c->nuv, kchunk);
    if (S < 1) S = 1;
    c->splits_simt = S;
    c->splits = S;
    dim3 grid(gp_cdiv(c->N, AB_N), gp_cdiv(c->N, AB_M), S);
    if (c->nuv == 0) {
        GP_CUDA(c, cudaMemsetAsync(c->gpart, 0, sizeof(float) * c->npix, c->stream));
        c->splits = 1;
        return GPAIR_OK;
    }
    k_adj_simt<<<grid, 256, 0, c->stream>>>(c->fx, c->fy, c->cw, c->N, c->nuv, kchunk, c->gpart);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

int gp_default_splits(int N, int nuv) { return adj_splits(N, nuv); }

// ------------------------------------------------------ gradient finalize

struct GradFinalizeArgs {
    const float *gpart;
    int splits, npix, mode;
    const float *img, *model;
    float alpha;
    int alpha_from_state;
    float *data_grad, *entropy_grad, *out;
    const float *g_old, *d;
    int dot_slot;
    double *partials;
    DevScalars *sc;
    FusedCtrl fc;
    int parts;  // threads per four pixels (a power of two); 1: one thread sums all splits
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void grad_finalize_body(const GradFinalizeArgs &A, const GpVGrid &vg)
{
    const float *__restrict__ gpart = A.gpart;
    const int splits = A.splits, npix = A.npix, mode = A.mode, dot_slot = A.dot_slot;
    const float *__restrict__ img = A.img;
    const float *__restrict__ model = A.model;
    float alpha = A.alpha;
    const int alpha_from_state = A.alpha_from_state;
    float *__restrict__ data_grad = A.data_grad;
    float *__restrict__ entropy_grad = A.entropy_grad;
    float *__restrict__ out = A.out;
    const float *__restrict__ g_old = A.g_old;
    const float *__restrict__ d = A.d;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ double smem[4 * 32];
    const double C = sc->adj_c, gscale = sc->gscale;
    const int reg_kind = sc->reg_kind;
    if (alpha_from_state) alpha = (float)sc->cg.alpha;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    // one pixel: the split sum in split order (FP64), then the gradient assembly
    auto finish = [&](int p, double g) {
        float gd = (float)(g * gscale - C);
        data_grad[p] = gd;
        if (mode == GRAD_FUSED) {
            float I = img[p], m = model[p];
            float eg = entropy_grad[p];
            eg = reg_grad(I, m, eg, reg_kind);
            entropy_grad[p] = eg;
            float fg = gd - alpha * eg;
            out[p] = fg;
            double fgd = fg, go = g_old[p], dd = d[p];
            acc[0] += fgd * fgd;
            acc[1] += fgd * go;
            acc[2] += fgd * dd;
            acc[3] += dd * go;
        }
    };
    // the split sum of pixels 4q .. 4q + 3 over splits [s0, s1), in split order (FP64)
    auto quad_sum = [&](int q, int nq, int s0, int s1, double (&g)[4]) {
        const float4 *g4 = reinterpret_cast<const float4 *>(gpart) + q;
        const size_t stride = (size_t)nq;
        int s = s0;
        for (; s + 8 <= s1; s += 8) {
            float4 a[8];
#pragma unroll
            for (int j = 0; j < 8; j++) a[j] = __ldcs(g4 + (size_t)(s + j) * stride);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                g[0] += a[j].x;
                g[1] += a[j].y;
                g[2] += a[j].z;
                g[3] += a[j].w;
            }
        }
        for (; s < s1; s++) {
            const float4 a = __ldcs(g4 + (size_t)s * stride);
            g[0] += a.x;
            g[1] += a.y;
            g[2] += a.z;
            g[3] += a.w;
        }
    };
    const int P = A.parts;
    if ((npix & 3) == 0 && P > 1) {
        // P threads per four pixels (small images: enough loads in flight to cover the
        // latency): part pp sums splits [pp S / P, (pp + 1) S / P); the parts are added
        // in part order through shared memory
        __shared__ double psum[GP_THREADS][4];
        const int nq = npix >> 2, qpb = blockDim.x / P;
        const int lq = threadIdx.x % qpb, pp = threadIdx.x / qpb;
        for (int qbase = vg.bx * qpb; qbase < nq; qbase += vg.nbx * qpb) {  // block-uniform
            const int q = qbase + lq;
            double g[4] = {0.0, 0.0, 0.0, 0.0};
            if (q < nq) quad_sum(q, nq, (pp * splits) / P, ((pp + 1) * splits) / P, g);
#pragma unroll
            for (int j = 0; j < 4; j++) psum[threadIdx.x][j] = g[j];
            __syncthreads();
            if (pp == 0 && q < nq) {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    double t = psum[lq][j];
                    for (int r = 1; r < P; r++) t += psum[r * qpb + lq][j];
                    finish(4 * q + j, t);
                }
            }
            __syncthreads();  // psum is rewritten by the next pass
        }
    } else if ((npix & 3) == 0) {
        // four consecutive pixels per thread: 16-byte loads, 8 splits (128 B) in flight
        const int nq = npix >> 2;
        for (int q = vg.bx * blockDim.x + threadIdx.x; q < nq; q += vg.nbx * blockDim.x) {
            double g[4] = {0.0, 0.0, 0.0, 0.0};
            quad_sum(q, nq, 0, splits, g);
#pragma unroll
            for (int j = 0; j < 4; j++) finish(4 * q + j, g[j]);
        }
    } else {
        for (int p = vg.bx * blockDim.x + threadIdx.x; p < npix; p += vg.nbx * blockDim.x) {
            double g = 0.0;
            int s = 0;
            for (; s + 16 <= splits; s += 16) {  // 16 loads in flight, summed in split order
                float a[16];
#pragma unroll
                for (int j = 0; j < 16; j++) a[j] = __ldcs(&gpart[(size_t)(s + j) * npix + p]);
#pragma unroll
                for (int j = 0; j < 16; j++) g += a[j];
            }
            for (; s < splits; s++) g += __ldcs(&gpart[(size_t)s * npix + p]);
            finish(p, g);
        }
    }
    if (mode != GRAD_FUSED) return;
    block_sum<4>(acc, smem);
    if (threadIdx.x == 0)
        for (int i = 0; i < 4; i++) partials[4 * vg.bx + i] = acc[i];
    if (last_block_of(&sc->counter[RED_GRAD], vg.nbx)) {
        double o[4];
        finish_sum<4>(partials, vg.nbx, o, smem);
        if (threadIdx.x == 0) {
            for (int i = 0; i < 4; i++) sc->grad_dots[dot_slot][i] = o[i];
            if (!isfinite(o[0])) sc->nonfinite |= 4u;
            sc->counter[RED_GRAD] = 0;
            run_fused_ctrl(sc, A.fc);
        }
    }
}

__global__ void __launch_bounds__(GP_THREADS) k_grad_finalize(const GradFinalizeArgs a)
{
    gp_pdl_enter();
    grad_finalize_body(a, gp_vgrid_hw());
}

struct GradFinalizeOp {
    using Args = GradFinalizeArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { grad_finalize_body(a, v); }
};

static GradFinalizeArgs grad_finalize_args(gpair_ctx *c, int which, int mode, float alpha, FusedCtrl fc)
{
    // alpha < 0 requests the value held in the device CG state (graph-captured runs)
    const int alpha_from_state = alpha < 0.f;
    const float *img = (which == GPAIR_IMG_TEMP) ? c->image_temp : c->image;
    float *out = (which == GPAIR_IMG_TEMP) ? c->grad_temp : c->full_grad_new;
    // one thread per pixel (per four pixels when the image size allows 16-byte loads);
    // for images too small to fill two waves of 148 SMs that way, up to c->gf_parts
    // threads per four pixels, each summing a contiguous part of the splits (contexts
    // that share the GPU keep one: their instances fill it together)
    int P = 1;
    const long long units = (c->npix & 3) == 0 ? c->npix / 4 : c->npix;
    if ((c->npix & 3) == 0)
        while (2 * P <= c->gf_parts && 2 * P <= c->splits && gp_cdiv(units * P, GP_THREADS) < 2 * 148) P *= 2;
    int g = gp_cdiv(units * P, GP_THREADS);
    if (g > GP_MAX_PARTIALS) g = GP_MAX_PARTIALS;
    if (g < 1) g = 1;
    GradFinalizeArgs a = {c->gpart, c->splits, c->npix, mode, img, c->model, alpha, alpha_from_state,
                          c->data_grad, c->entropy_grad, out, c->full_grad, c->descent_dir,
                          which == GPAIR_IMG_TEMP ? 1 : 0, slot_partials(c, RED_GRAD), c->sc, fc, P, g, 1};
    return a;
}

int gp_grad_finalize(gpair_ctx *c, int which, int mode, float alpha)
{
    const GradFinalizeArgs a = grad_finalize_args(c, which, mode, alpha, take_fused_ctrl(c));
    GP_LAUNCH(c, gp_launch(c, k_grad_finalize, dim3(a.nbx), dim3(GP_THREADS), 0, a));
    return GPAIR_OK;
}

// entropy gradient alone (gpu_compute_entropy_gradient, kernel_entropy_gs_grad.cl)
__global__ void k_entropy_grad(const float *__restrict__ img, const float *__restrict__ model, int npix,
                               float *__restrict__ eg, const DevScalars *__restrict__ sc)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    eg[p] = reg_grad(img[p], model[p], eg[p], sc->reg_kind);
}

int gp_entropy_gradient(gpair_ctx *c, int which)
{
    const float *img = (which == GPAIR_IMG_TEMP) ? c->image_temp : c->image;
    k_entropy_grad<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(img, c->model, c->npix, c->entropy_grad, c->sc);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// criterion gradient alone (kernel_criterion_grad.cl)
__global__ void k_crit_grad(const float *__restrict__ dg, const float *__restrict__ eg, float alpha, int npix,
                            float *__restrict__ out)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < npix) out[p] = dg[p] - alpha * eg[p];
}

int gp_criterion_gradient(gpair_ctx *c, float alpha, float *out)
{
    k_crit_grad<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(c->data_grad, c->entropy_grad, alpha, c->npix, out);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// -------------------------------------------------------------- CG vectors

__global__ void __launch_bounds__(GP_THREADS) k_dot(const float *__restrict__ a, const float *__restrict__ b, int n,
                                                    double *__restrict__ partials, DevScalars *__restrict__ sc)
{
    __shared__ double smem[32];
    double acc[1] = {0.0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        acc[0] += (double)a[p] * (double)b[p];
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
    if (last_block(&sc->counter[RED_DOT])) {
        double o[1];
        finish_sum<1>(partials, gridDim.x, o, smem);
        if (threadIdx.x == 0) {
            sc->dot = o[0];
            sc->dot_f = (float)o[0];
            sc->counter[RED_DOT] = 0;
        }
    }
}

int gp_dot(gpair_ctx *c, const float *a, const float *b, int n)
{
    k_dot<<<red_grid(n), GP_THREADS, 0, c->stream>>>(a, b, n, slot_partials(c, RED_DOT), c->sc);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// d = beta d - g_new, and d.g_new (FP64)
struct DescentArgs {
    float *d;
    const float *g;
    int n, beta_from_state;
    double beta_host;
    double *partials;
    DevScalars *sc;
    FusedCtrl fc;
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void descent_body(const DescentArgs &A, const GpVGrid &vg)
{
    float *__restrict__ d = A.d;
    const float *__restrict__ g = A.g;
    const int n = A.n;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ double smem[32];
    const double beta = A.beta_from_state ? sc->cg.beta : A.beta_host;
    double acc[1] = {0.0};
    for (int p = vg.bx * blockDim.x + threadIdx.x; p < n; p += vg.nbx * blockDim.x) {
        // beta = 0 (first iteration, restarts) must not read the old direction:
        // 0 * d_old is NaN when a previous run left non-finite values there
        float dn = beta != 0.0 ? (float)(beta * (double)d[p] - (double)g[p]) : -g[p];
        d[p] = dn;
        acc[0] += (double)dn * (double)g[p];
    }
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) partials[vg.bx] = acc[0];
    if (last_block_of(&sc->counter[RED_DIR], vg.nbx)) {
        double o[1];
        finish_sum<1>(partials, vg.nbx, o, smem);
        if (threadIdx.x == 0) {
            sc->dir_dot = o[0];
            sc->counter[RED_DIR] = 0;
            run_fused_ctrl(sc, A.fc);
        }
    }
}

__global__ void __launch_bounds__(GP_THREADS) k_descent(const DescentArgs a)
{
    gp_pdl_enter();
    descent_body(a, gp_vgrid_hw());
}

struct DescentOp {
    using Args = DescentArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { descent_body(a, v); }
};

static DescentArgs descent_args(gpair_ctx *c, int beta_from_state, double beta_host, FusedCtrl fc)
{
    DescentArgs a = {c->descent_dir, c->full_grad_new, c->npix, beta_from_state, beta_host,
                     slot_partials(c, RED_DIR), c->sc, fc, red_grid(c->npix), 1};
    return a;
}

int gp_descent_dir(gpair_ctx *c, int beta_from_state, double beta_host)
{
    const DescentArgs a = descent_args(c, beta_from_state, beta_host, take_fused_ctrl(c));
    GP_LAUNCH(c, gp_launch(c, k_descent, dim3(a.nbx), dim3(GP_THREADS), 0, a));
    return GPAIR_OK;
}

// ------------------------------------------------ projected L-BFGS (method 4)
//
// No counterpart in the reference (its methods are the CG beta rules of
// gpair1/trunk/gpair.c:733-753). Pixels on the positivity bound whose gradient
// points outward are held fixed (q = g elsewhere, 0 there; the direction is 0
// there too). The direction is the compact form of the inverse BFGS matrix
// (Byrd, Nocedal and Schnabel, 1994) over the newest GP_LB_PAIRS pairs
// s = x_new - x_old (the step taken, after the clamp), y = g_new - g_old:
//   d = -(gamma q + S^T t - gamma Y^T R^-1 u),  u = S q,
//   t = R^-T ((D + gamma Y Y^T) R^-1 u - gamma Y q),
// R = upper triangle of S Y^T, D its diagonal, gamma = s.y / y.y of the newest
// pair. The device needs three passes per iteration: the candidate pair and
// its dots with the stored pairs, the 2m + 1 dots of q, and one combination
// pass; the m x m algebra runs in the controller in FP64.

__device__ __forceinline__ bool lb_fixed(float I, float g, double minvalue)
{
    return (double)I <= minvalue * 1.000001 && g > 0.f;
}

// Candidate pair (s, y) of the last step into the free buffer, with its dots
// s.y, y.y, s.s and s_i.y, y_i.y against the stored pairs i (logical order).
// Without a valid previous image (first iteration) it writes and sums nothing.
__global__ void __launch_bounds__(GP_THREADS) k_lbfgs_pair(const float *__restrict__ img,
                                                           const float *__restrict__ xold,
                                                           const float *__restrict__ gnew,
                                                           const float *__restrict__ gold, float *__restrict__ S,
                                                           float *__restrict__ Y, int n, double *__restrict__ partials,
                                                           DevScalars *__restrict__ sc, FusedCtrl fc)
{
    gp_pdl_enter();
    __shared__ double smem[GP_LB_NPD * 32];
    const CgState &cs = sc->cg;
    const int active = cs.lb_xvalid;
    const int m = cs.lb_count;
    float *sn = S + (size_t)cs.lb_slot[GP_LB_PAIRS] * n, *yn = Y + (size_t)cs.lb_slot[GP_LB_PAIRS] * n;
    const float *si[GP_LB_PAIRS], *yi[GP_LB_PAIRS];
#pragma unroll
    for (int i = 0; i < GP_LB_PAIRS; i++) {
        si[i] = S + (size_t)cs.lb_slot[i] * n;
        yi[i] = Y + (size_t)cs.lb_slot[i] * n;
    }
    double acc[GP_LB_NPD];
#pragma unroll
    for (int k = 0; k < GP_LB_NPD; k++) acc[k] = 0.0;
    if (active) {
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
            const float s = img[p] - xold[p], y = gnew[p] - gold[p];
            sn[p] = s;
            yn[p] = y;
            const double sd = s, yd = y;
            acc[0] += sd * yd;
            acc[1] += yd * yd;
            acc[2] += sd * sd;
#pragma unroll
            for (int i = 0; i < GP_LB_PAIRS; i++) {
                if (i < m) {
                    acc[3 + i] += (double)si[i][p] * yd;
                    acc[3 + GP_LB_PAIRS + i] += (double)yi[i][p] * yd;
                }
            }
        }
    }
    block_sum<GP_LB_NPD>(acc, smem);
    if (threadIdx.x == 0)
        for (int k = 0; k < GP_LB_NPD; k++) partials[(size_t)blockIdx.x * GP_LB_NPD + k] = acc[k];
    if (last_block(&sc->counter[RED_LBP])) {
        double o[GP_LB_NPD];
        finish_sum<GP_LB_NPD>(partials, gridDim.x, o, smem);
        if (threadIdx.x == 0) {
            for (int k = 0; k < GP_LB_NPD; k++) sc->lb_pdots[k] = o[k];
            sc->counter[RED_LBP] = 0;
            run_fused_ctrl(sc, fc);
        }
    }
}

// q = projected gradient; q.q, s_i.q, y_i.q over the stored pairs
__global__ void __launch_bounds__(GP_THREADS) k_lbfgs_dots(const float *__restrict__ img, const float *__restrict__ g,
                                                           const float *__restrict__ S, const float *__restrict__ Y,
                                                           int n, double *__restrict__ partials,
                                                           DevScalars *__restrict__ sc, FusedCtrl fc)
{
    gp_pdl_enter();
    __shared__ double smem[GP_LB_NQD * 32];
    const CgState &cs = sc->cg;
    const int m = cs.lb_count;
    const double minvalue = cs.minvalue;
    const float *si[GP_LB_PAIRS], *yi[GP_LB_PAIRS];
#pragma unroll
    for (int i = 0; i < GP_LB_PAIRS; i++) {
        si[i] = S + (size_t)cs.lb_slot[i] * n;
        yi[i] = Y + (size_t)cs.lb_slot[i] * n;
    }
    double acc[GP_LB_NQD];
#pragma unroll
    for (int k = 0; k < GP_LB_NQD; k++) acc[k] = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float gp = g[p];
        if (lb_fixed(img[p], gp, minvalue)) continue;
        const double q = gp;
        acc[0] += q * q;
#pragma unroll
        for (int i = 0; i < GP_LB_PAIRS; i++) {
            if (i < m) {
                acc[1 + i] += (double)si[i][p] * q;
                acc[1 + GP_LB_PAIRS + i] += (double)yi[i][p] * q;
            }
        }
    }
    block_sum<GP_LB_NQD>(acc, smem);
    if (threadIdx.x == 0)
        for (int k = 0; k < GP_LB_NQD; k++) partials[(size_t)blockIdx.x * GP_LB_NQD + k] = acc[k];
    if (last_block(&sc->counter[RED_LBD])) {
        double o[GP_LB_NQD];
        finish_sum<GP_LB_NQD>(partials, gridDim.x, o, smem);
        if (threadIdx.x == 0) {
            for (int k = 0; k < GP_LB_NQD; k++) sc->lb_qdots[k] = o[k];
            if (!isfinite(o[0])) sc->nonfinite |= 4u;
            sc->counter[RED_LBD] = 0;
            run_fused_ctrl(sc, fc);
        }
    }
}

// d = -(cq q + sum cs_i s_i + sum cy_i y_i) on free pixels, 0 on fixed ones;
// x_old = image; d.g and max |d|
__global__ void __launch_bounds__(GP_THREADS) k_lbfgs_combine(const float *__restrict__ img,
                                                              const float *__restrict__ g,
                                                              const float *__restrict__ S,
                                                              const float *__restrict__ Y, float *__restrict__ d,
                                                              float *__restrict__ xold, int n,
                                                              double *__restrict__ partials,
                                                              DevScalars *__restrict__ sc, FusedCtrl fc)
{
    gp_pdl_enter();
    __shared__ double smem[32];
    const CgState &cs = sc->cg;
    const int m = cs.lb_count;
    const double minvalue = cs.minvalue, cq = cs.lb_cq;
    const float *si[GP_LB_PAIRS], *yi[GP_LB_PAIRS];
    double ca[GP_LB_PAIRS], cb[GP_LB_PAIRS];
#pragma unroll
    for (int i = 0; i < GP_LB_PAIRS; i++) {
        si[i] = S + (size_t)cs.lb_slot[i] * n;
        yi[i] = Y + (size_t)cs.lb_slot[i] * n;
        ca[i] = cs.lb_cs[i];
        cb[i] = cs.lb_cy[i];
    }
    double acc[1] = {0.0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float I = img[p], gp = g[p];
        xold[p] = I;
        float dn = 0.f;
        if (!lb_fixed(I, gp, minvalue)) {
            double h = cq * (double)gp;
#pragma unroll
            for (int i = 0; i < GP_LB_PAIRS; i++)
                if (i < m) h += ca[i] * (double)si[i][p] + cb[i] * (double)yi[i][p];
            dn = (float)(-h);
        }
        d[p] = dn;
        acc[0] += (double)dn * (double)gp;
    }
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
    if (last_block(&sc->counter[RED_DIR])) {
        double o[1];
        finish_sum<1>(partials, gridDim.x, o, smem);
        if (threadIdx.x == 0) {
            sc->dir_dot = o[0];
            sc->counter[RED_DIR] = 0;
            run_fused_ctrl(sc, fc);
        }
    }
}

int gp_lbfgs_alloc(gpair_ctx *c)
{
    if (c->lb_s) return GPAIR_OK;
    const size_t n = (size_t)(GP_LB_PAIRS + 1) * c->npix;
    GP_CUDA(c, cudaMalloc(&c->lb_s, n * sizeof(float)));
    GP_CUDA(c, cudaMalloc(&c->lb_y, n * sizeof(float)));
    GP_CUDA(c, cudaMalloc(&c->lb_xold, (size_t)c->npix * sizeof(float)));
    GP_CUDA(c, cudaMemsetAsync(c->lb_s, 0, n * sizeof(float), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->lb_y, 0, n * sizeof(float), c->stream));
    GP_CUDA(c, cudaMemsetAsync(c->lb_xold, 0, (size_t)c->npix * sizeof(float), c->stream));
    return GPAIR_OK;
}

void gp_lbfgs_free(gpair_ctx *c)
{
    if (c->lb_s) cudaFree(c->lb_s);
    if (c->lb_y) cudaFree(c->lb_y);
    if (c->lb_xold) cudaFree(c->lb_xold);
    c->lb_s = c->lb_y = c->lb_xold = nullptr;
}

// The direction of one iteration: candidate pair (controller: accept / drop),
// dots of the projected gradient (controller: coefficients), combination
// (controller: the line-search start, as after the CG descent update). The
// controller steps run fused into the last block of each pass; the caller
// sets the first one (CTRL_LB_PAIR) in c->fuse_ctrl.
int gp_lbfgs_direction(gpair_ctx *c)
{
    const int last = c->fuse_ctrl;  // the controller step after the direction (CTRL_AFTER_DIR)
    int rc = gp_lbfgs_alloc(c);
    if (rc) return rc;
    const int g = red_grid(c->npix);
    c->fuse_ctrl = CTRL_LB_PAIR;
    GP_LAUNCH(c, gp_launch(c, k_lbfgs_pair, dim3(g), dim3(GP_THREADS), 0, c->image, c->lb_xold, c->full_grad_new,
                           c->full_grad, c->lb_s, c->lb_y, c->npix, slot_partials(c, RED_LBP), c->sc,
                           take_fused_ctrl(c)));
    c->fuse_ctrl = CTRL_LB_COEF;
    GP_LAUNCH(c, gp_launch(c, k_lbfgs_dots, dim3(g), dim3(GP_THREADS), 0, c->image, c->full_grad_new, c->lb_s,
                           c->lb_y, c->npix, slot_partials(c, RED_LBD), c->sc, take_fused_ctrl(c)));
    c->fuse_ctrl = last;
    GP_LAUNCH(c, gp_launch(c, k_lbfgs_combine, dim3(g), dim3(GP_THREADS), 0, c->image, c->full_grad_new, c->lb_s,
                           c->lb_y, c->descent_dir, c->lb_xold, c->npix, slot_partials(c, RED_DIR), c->sc,
                           take_fused_ctrl(c)));
    return GPAIR_OK;
}

// image = max(image + s d, minval); optionally full_grad = full_grad_new
struct UpdateImageArgs {
    float *img;
    const float *d;
    int n, step_from_state;
    double step_host, minval;
    const float *gnew;
    float *gold;
    const DevScalars *sc;
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void update_image_body(const UpdateImageArgs &A, const GpVGrid &vg)
{
    float *__restrict__ img = A.img;
    const float *__restrict__ d = A.d;
    const float *__restrict__ gnew = A.gnew;
    float *__restrict__ gold = A.gold;
    const int n = A.n;
    const double s = A.step_from_state ? A.sc->cg.sel : A.step_host;
    const double minval = A.step_from_state ? A.sc->cg.minvalue : A.minval;
    for (int p = vg.bx * blockDim.x + threadIdx.x; p < n; p += vg.nbx * blockDim.x) {
        double t = (double)img[p] + s * (double)d[p];
        if (t < minval) t = minval;
        img[p] = (float)t;
        if (gold) gold[p] = gnew[p];
    }
}

__global__ void __launch_bounds__(256) k_update_image(const UpdateImageArgs a)
{
    gp_pdl_enter();
    update_image_body(a, gp_vgrid_hw());
}

struct UpdateImageOp {
    using Args = UpdateImageArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { update_image_body(a, v); }
};

static UpdateImageArgs update_image_args(gpair_ctx *c, int step_from_state, double step_host, double minval,
                                         int backup)
{
    UpdateImageArgs a = {c->image, c->descent_dir, c->npix, step_from_state, step_host, minval, c->full_grad_new,
                         backup ? c->full_grad : nullptr, c->sc, gp_cdiv(c->npix, 256), 1};
    return a;
}

int gp_update_image(gpair_ctx *c, int step_from_state, double step_host, double minval, int backup)
{
    const UpdateImageArgs a = update_image_args(c, step_from_state, step_host, minval, backup);
    GP_LAUNCH(c, gp_launch(c, k_update_image, dim3(a.nbx), dim3(256), 0, a));
    return GPAIR_OK;
}

// temp = image + s d (clamped at minval when clamp != 0), float arithmetic of
// kernel_update_tempimage.cl / kernel_criterion_step.cl
__global__ void k_update_temp(const float *__restrict__ img, const float *__restrict__ d, int n, float s,
                              float minval, int clamp, float *__restrict__ temp)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float t = img[p] + s * d[p];
    if (clamp && t < minval) t = minval;
    temp[p] = t;
}

int gp_update_temp(gpair_ctx *c, double step, double minval, int clamp)
{
    k_update_temp<<<gp_cdiv(c->npix, 256), 256, 0, c->stream>>>(c->image, c->descent_dir, c->npix, (float)step,
                                                                (float)minval, clamp, c->image_temp);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// ------------------------------------------- batched line-search trials

// GP_NTR trial images I_j = max(I + s_j d, minval) (s_j = cg.ts[j], blockIdx.y
// = j), each with its flux and regulariser summed in FP64 (the trial part of
// kernel_update_tempimage.cl + kernel_entropy_gs.cl, for a whole batch), for
// the CUDA-core forward; the tensor path prepares its trials row by row
// together with their operands (k_tc_prep_rows).
__global__ void __launch_bounds__(GP_THREADS) k_trials_prep(const float *__restrict__ img,
                                                            const float *__restrict__ d, float *__restrict__ trials,
                                                            const float *__restrict__ model, int npix,
                                                            double *__restrict__ partials,
                                                            DevScalars *__restrict__ sc, const int *__restrict__ gate)
{
    __shared__ double smem[2 * 32];
    if (gate && !*gate) return;  // lockstep batches: this instance's line search is over
    const int j = blockIdx.y;
    const double s = sc->cg.ts[j], minval = sc->cg.minvalue;
    float *dst = trials + (size_t)j * npix;
    double acc[2] = {0.0, 0.0};
    const int reg_kind = sc->reg_kind;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        double t = (double)img[p] + s * (double)d[p];
        if (t < minval) t = minval;
        const float I = (float)t;
        dst[p] = I;
        const double Id = I, m = model[p];
        acc[0] += Id;
        acc[1] += reg_term(Id, m, reg_kind);
    }
    block_sum<2>(acc, smem);
    double *pp = partials + (size_t)j * gridDim.x * 2;
    if (threadIdx.x == 0) {
        pp[2 * blockIdx.x] = acc[0];
        pp[2 * blockIdx.x + 1] = acc[1];
    }
    if (last_block(&sc->t_counter[j])) {
        double o[2];
        finish_sum<2>(pp, gridDim.x, o, smem);
        if (threadIdx.x == 0) {
            sc->t_flux[j] = o[0];
            sc->t_invflux[j] = 1.0 / o[0];
            sc->t_entropy[j] = o[1];
            sc->t_counter[j] = 0;
        }
    }
}

// chi2 of every trial of a batch (blockIdx.y = trial): V = (sum of the trial's
// epp partial entries) / F_j, then V2 and T3 residuals as in k_vis_data; mock
// data and adjoint weights are not needed for trials. The last block of the
// whole grid sums each trial's partials in block order and runs the controller.
struct VisChi2BatchArgs {
    const float2 *vpart;
    int epp, nuv, npow, nbis;
    const float *data, *data_err;
    const int4 *tri;
    const float2 *phasor;
    double *partials;
    DevScalars *sc;
    FusedCtrl fc;
    const int *gate;
    const double2 *visb;  // the trials' visibilities summed beforehand (k_vis_sum_batch), or null
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void vis_chi2_batch_body(const VisChi2BatchArgs &A, const GpVGrid &vg)
{
    const float2 *__restrict__ vpart = A.vpart;
    const int epp = A.epp, nuv = A.nuv, npow = A.npow, nbis = A.nbis;
    const float *__restrict__ data = A.data;
    const float *__restrict__ data_err = A.data_err;
    const int4 *__restrict__ tri = A.tri;
    const float2 *__restrict__ phasor = A.phasor;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ double smem[32];
    if (A.gate && !*A.gate) return;  // lockstep batches: this instance's line search is over
    const int j = vg.by;
    const double invF = sc->t_invflux[j];
    const float2 *vp = vpart + (size_t)j * epp * nuv;
    const double2 *vb = A.visb ? A.visb + (size_t)j * nuv : nullptr;
#define VIS_B(k) (vb ? vb[(k)] : sum_vpart(vp, epp, nuv, (k), invF))
    double chi[1] = {0.0};
    const int nitems = npow + nbis;
    for (int i = vg.bx * blockDim.x + threadIdx.x; i < nitems; i += vg.nbx * blockDim.x) {
        if (i < npow) {
            double2 V = VIS_B(i);
            double m2 = V.x * V.x + V.y * V.y;
            double r = (m2 - (double)data[i]) * data_err[i];
            chi[0] += r * r;
        } else {
            const int t = i - npow;
            int4 q = tri[t];
            double2 va = VIS_B(q.x);
            double2 vbb = VIS_B(q.y);
            double2 vc = VIS_B(q.z);
            if (q.w & 1) va = cconj(va);
            if (q.w & 2) vbb = cconj(vbb);
            if (q.w & 4) vc = cconj(vc);
            float2 phf = phasor[t];
            double2 t3 = cmul(cmul(cmul(va, vbb), vc), make_double2(phf.x, phf.y));
            const int r0 = npow + 2 * t;
            double rre = (t3.x - (double)data[r0]) * data_err[r0];
            double rim = (t3.y - (double)data[r0 + 1]) * data_err[r0 + 1];
            chi[0] += rre * rre + rim * rim;
        }
    }
    block_sum<1>(chi, smem);
    if (threadIdx.x == 0) partials[(size_t)j * vg.nbx + vg.bx] = chi[0];
    if (last_block_of(&sc->t_counter[GP_NTR], vg.nbx * vg.nby)) {
        // one warp per trial, all trials at once; fixed lane order and shuffle tree
        const int lane = threadIdx.x & 31;
        for (int jj = threadIdx.x >> 5; jj < vg.nby; jj += blockDim.x >> 5) {
            const double *pp = partials + (size_t)jj * vg.nbx;
            double v = 0.0;
            for (int b = lane; b < vg.nbx; b += 32) v += __ldcg(&pp[b]);
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) sc->t_chi2[jj] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            sc->t_counter[GP_NTR] = 0;
            run_fused_ctrl(sc, A.fc);
        }
    }
}

#undef VIS_B

// the trials' visibilities V_jk = (sum of trial j's partial entries) / F_j into visb,
// summed once instead of once per gathering triangle vertex (the same sum)
__global__ void __launch_bounds__(GP_THREADS) k_vis_sum_batch(const float2 *__restrict__ vpart, int epp, int nuv,
                                                              const DevScalars *__restrict__ sc,
                                                              double2 *__restrict__ visb,
                                                              const int *__restrict__ gate)
{
    gp_pdl_enter();
    if (gate && !*gate) return;  // lockstep batches: this instance's line search is over
    const int j = blockIdx.y;
    const double invF = sc->t_invflux[j];
    const float2 *vp = vpart + (size_t)j * epp * nuv;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nuv; k += gridDim.x * blockDim.x)
        visb[(size_t)j * nuv + k] = sum_vpart(vp, epp, nuv, k, invF);
}

__global__ void __launch_bounds__(GP_THREADS) k_vis_chi2_batch(const VisChi2BatchArgs a)
{
    gp_pdl_enter();
    vis_chi2_batch_body(a, gp_vgrid_hw());
}

struct VisChi2BatchOp {
    using Args = VisChi2BatchArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { vis_chi2_batch_body(a, v); }
};

// Blocks per trial: at most one wave of resident blocks over the whole batch
// (a partial second wave would leave most SMs idle while it runs), at most 256
// (the per-trial partial-sum area), at least one.
static int batch_blocks_per_trial(gpair_ctx *c)
{
    int g = gp_cdiv(c->npix, GP_THREADS * 2);
    if (g > c->batch_wave[0]) g = c->batch_wave[0];
    if (g > 256) g = 256;
    return g < 1 ? 1 : g;
}

static int batch_wave_blocks(const void *kernel, int nsm)
{
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, GP_THREADS, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int w = per_sm * nsm / GP_NTR;
    return w < 1 ? 1 : w;
}

int gp_batch_alloc(gpair_ctx *c)
{
    int epp_tc = 0;
    if (c->precision != GPAIR_PREC_FP32) {
        // every time: the tensor state (and its trial operand stack) is rebuilt when
        // the precision or the tile layout changes, the trial images are not
        int rc = gp_tc_batch_prepare(c, &epp_tc);
        if (rc) return rc;
    }
    if (c->image_trials) return GPAIR_OK;
    const int mt_simt = gp_cdiv(c->N, FB_M);
    const int epp_max = mt_simt > epp_tc ? mt_simt : epp_tc;
    GP_CUDA(c, cudaMalloc(&c->image_trials, sizeof(float) * (size_t)GP_NTR * c->npix));
    GP_CUDA(c, cudaMalloc(&c->vpart_b, sizeof(float2) * (size_t)GP_NTR * epp_max * (c->nuv ? c->nuv : 1)));
    GP_CUDA(c, cudaMalloc(&c->partials_b, sizeof(double) * (size_t)GP_NTR * 1024 * 2));
    if (epp_max > VIS_PRESUM_ENTRIES)
        GP_CUDA(c, cudaMalloc(&c->visb, sizeof(double2) * (size_t)GP_NTR * (c->nuv ? c->nuv : 1)));
    int nsm = 148;
    GP_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    c->batch_wave[0] = batch_wave_blocks((const void *)k_trials_prep, nsm);
    c->batch_wave[1] = batch_wave_blocks((const void *)k_vis_chi2_batch, nsm);
    return GPAIR_OK;
}

void gp_batch_free(gpair_ctx *c)
{
    if (c->image_trials) c->buf_gen++;
    if (c->image_trials) cudaFree(c->image_trials);
    if (c->vpart_b) cudaFree(c->vpart_b);
    if (c->partials_b) cudaFree(c->partials_b);
    if (c->visb) cudaFree(c->visb);
    c->image_trials = nullptr;
    c->vpart_b = nullptr;
    c->partials_b = nullptr;
    c->visb = nullptr;
}

int gp_trials_prep_launch(gpair_ctx *c)
{
    dim3 g(batch_blocks_per_trial(c), GP_NTR);
    k_trials_prep<<<g, GP_THREADS, 0, c->stream>>>(c->image, c->descent_dir, c->image_trials, c->model, c->npix,
                                                   c->partials_b, c->sc, c->gate);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// chi2 of the GP_NTR trials of a batch from their partial visibilities (epp
// entries per trial), then the fused controller
// presum: read the visibilities from visb (k_vis_sum_batch runs first) when the
// partial entries are many; grouped launches pass 0
static VisChi2BatchArgs batch_chi2_args(gpair_ctx *c, int epp, FusedCtrl fc, const int *gate, int presum = 0)
{
    int nb = gp_cdiv(c->npow + c->nbis, GP_THREADS * 2);
    if (nb > c->batch_wave[1]) nb = c->batch_wave[1];  // one wave over the batch
    if (nb > 1024) nb = 1024;
    if (nb < 1) nb = 1;
    const double2 *vb = (presum && epp > VIS_PRESUM_ENTRIES && c->visb) ? c->visb : nullptr;
    VisChi2BatchArgs a = {c->vpart_b, epp, c->nuv, c->npow, c->nbis, c->data, c->data_err, c->tri, c->phasor,
                          c->partials_b, c->sc, fc, gate, vb, nb, GP_NTR};
    return a;
}

static int batch_chi2(gpair_ctx *c, int epp)
{
    const VisChi2BatchArgs a = batch_chi2_args(c, epp, take_fused_ctrl(c), c->gate, 1);
    if (a.visb) {
        int nb = gp_cdiv(c->nuv, GP_THREADS);
        if (nb > 148) nb = 148;  // 8 trials: about eight blocks per SM
        GP_LAUNCH(c, gp_launch(c, k_vis_sum_batch, dim3(nb, GP_NTR), dim3(GP_THREADS), 0, (const float2 *)c->vpart_b,
                               epp, c->nuv, (const DevScalars *)c->sc, c->visb, c->gate));
    }
    GP_LAUNCH(c, gp_launch(c, k_vis_chi2_batch, dim3(a.nbx, a.nby), dim3(GP_THREADS), 0, a));
    return GPAIR_OK;
}

// One batched evaluation: GP_NTR trial images -> forward DFTs -> chi2 of each,
// then the controller (fused into the last block of the chi2 kernel). With
// `ev` (4 events) the stage boundaries are recorded on the stream.
static int eval_batch(gpair_ctx *c, cudaEvent_t *ev)
{
    int rc = gp_batch_alloc(c);
    if (rc) return rc;
    int epp;
    if (ev) cudaEventRecord(ev[0], c->stream);
    gp_stage_begin(c, 0);
    if (c->precision != GPAIR_PREC_FP32) {
        if ((rc = gp_tc_trials_prep_split(c, c->partials_b))) return rc;
        gp_stage_end(c);
        if (ev) cudaEventRecord(ev[1], c->stream);
        gp_stage_begin(c, 1);
        if ((rc = gp_tc_forward_batch_gemm(c))) return rc;
        epp = c->epp;
    } else {
        if ((rc = gp_trials_prep_launch(c))) return rc;
        gp_stage_end(c);
        if (ev) cudaEventRecord(ev[1], c->stream);
        gp_stage_begin(c, 1);
        epp = gp_cdiv(c->N, FB_M);
        dim3 grid(gp_cdiv(c->nuv, FB_K), epp, GP_NTR);
        k_fwd_simt<<<grid, 256, 0, c->stream>>>(c->image_trials, c->fx, c->fy, c->N, c->nuv, c->vpart_b, c->gate);
        GP_LAUNCH_CHECK(c);
    }
    gp_stage_end(c);
    if (ev) cudaEventRecord(ev[2], c->stream);
    gp_stage_begin(c, 2);
    if ((rc = batch_chi2(c, epp))) return rc;
    gp_stage_end(c);
    if (ev) cudaEventRecord(ev[3], c->stream);
    return GPAIR_OK;
}

// The parts of a batched evaluation around its forward, for lockstep batches
// whose forwards run as one grouped launch (tensor path): 1 = trial images and
// operands, 2 = chi2 of each trial and the controller.
int gp_eval_batch_part(gpair_ctx *c, int part)
{
    int rc = gp_batch_alloc(c);
    if (rc) return rc;
    if (c->precision == GPAIR_PREC_FP32) return GPAIR_ERR_STATE;
    if (part == 1) return gp_tc_trials_prep_split(c, c->partials_b);
    if ((rc = gp_tc_batch_prepare(c, nullptr))) return rc;
    return batch_chi2(c, c->epp);
}

int gp_eval_batch(gpair_ctx *c) { return eval_batch(c, nullptr); }
int gp_eval_batch_timed(gpair_ctx *c, cudaEvent_t *ev) { return eval_batch(c, ev); }

// --------------------------------------------- single-pixel update

// One pixel changes from I_old to `value`: the total flux, the regulariser
// sum and the image are updated on one thread; V follows in k_update_pixel_vis.
// Corrected form of the reference's single-pixel flux change
// (gpair1/trunk/cpu.c:477-486, gpair1/trunk/gpu.c:2137-2182): with the total
// flux going from F to F' = F + delta, V'_k = (F V_k + delta e_k(x, y)) / F'.
__global__ void k_update_pixel_scalar(float *__restrict__ img, const float *__restrict__ model, int p, float value,
                                      DevScalars *__restrict__ sc)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double old = img[p], nv = value, m = model[p];
    const double F = sc->flux, Fn = F + (nv - old);
    sc->upd_flux_old = F;
    sc->upd_delta = nv - old;
    sc->flux = Fn;
    sc->invflux = 1.0 / Fn;
    sc->flux_f = (float)Fn;
    sc->invflux_f = (float)(1.0 / Fn);
    sc->entropy += reg_term(nv, m, sc->reg_kind) - reg_term(old, m, sc->reg_kind);
    sc->entropy_f = (float)sc->entropy;
    sc->imax = fmax(sc->imax, fabs(nv));
    img[p] = value;
}

__global__ void k_update_pixel_vis(const float2 *__restrict__ fx, const float2 *__restrict__ fy, int N, int nuv,
                                   int x, int y, double2 *__restrict__ visd, const DevScalars *__restrict__ sc)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nuv) return;
    const float2 a = fx[(size_t)k * N + x], b = fy[(size_t)k * N + y];
    const double er = (double)a.x * b.x - (double)a.y * b.y, ei = (double)a.x * b.y + (double)a.y * b.x;
    const double F = sc->upd_flux_old, d = sc->upd_delta, inv = sc->invflux;
    const double2 V = visd[k];
    visd[k] = make_double2((F * V.x + d * er) * inv, (F * V.y + d * ei) * inv);
}

int gp_update_pixel(gpair_ctx *c, int x, int y, float value)
{
    const int p = x + y * c->N;
    k_update_pixel_scalar<<<1, 32, 0, c->stream>>>(c->image, c->model, p, value, c->sc);
    GP_LAUNCH_CHECK(c);
    if (c->nuv) {
        k_update_pixel_vis<<<gp_cdiv(c->nuv, 256), 256, 0, c->stream>>>(c->fx, c->fy, c->N, c->nuv, x, y, c->visd,
                                                                       c->sc);
        GP_LAUNCH_CHECK(c);
    }
    c->fuse_ctrl = -1;
    return vis_data_launch(c, 1);  // V2, T3, chi2 and the adjoint weights from the updated V
}

// ------------------------------------------------------- CG controller

__device__ void cg_zoom_next(CgState &s)
{
    // top of the zoom loop, gpair1/trunk/gpu.c:1977-1990
    if (s.zoom_counter > 0 && (s.z_J_old - s.J_init - s.wolfe1 * s.z_s_old) != 0.0)
        s.z_s = fabs(s.wolfe1 * s.z_s_old * s.z_s_old / (2.0 * (s.z_J_old - s.J_init - s.wolfe1 * s.z_s_old)));
    if (s.zoom_counter == 0 || s.z_s < s.lo || s.z_s > s.hi) s.z_s = (s.hi - s.lo) / 2.0 + s.lo;
    if (fabs(s.hi - s.lo) < 1e-14 || s.zoom_trials >= s.max_zoom) {
        s.sel = s.lo;
        s.action = CG_DONE;
        return;
    }
    s.s = s.z_s;
    s.zoom_trials++;
    s.action = CG_EVAL_CRIT;
}

__device__ void cg_zoom_enter(CgState &s, double lo, double hi, double J_lo)
{
    s.phase = CG_PH_ZOOM;
    s.lo = lo;
    s.hi = hi;
    s.J_lo = J_lo;
    s.z_s = 0.0;
    s.z_s_old = 0.0;
    s.z_J_old = 0.0;
    s.zoom_counter = 0;
    s.zoom_trials = 0;
    cg_zoom_next(s);
}

// Batched line search: a grid of GP_NTR steps s_c R^(j-3), R = GP_LS_RATIO
__device__ void ls_batch_grid(CgState &s)
{
    for (int j = 0; j < GP_NTR; j++) {
        double t = ldexp(s.s_c, GP_LS_RATIO_LOG2 * (j - 3));  // s_c 4^(j-3), exact
        s.ts[j] = t < s.batch_step_max ? t : s.batch_step_max;
    }
    s.action = CG_EVAL_BATCH;
}

__device__ void ls_batch_accept(CgState &s, double sb, double Jb)
{
    s.sel = sb;
    s.Jt = Jb;
    if (sb > 0.0) s.s_c = sb;
    s.action = CG_DONE;
}

// After a batch: record its points, then shift the grid (no decrease yet, or
// the best step is the largest tried), refine inside the bracket of the best
// point, or accept the best point.
__device__ void ls_batch_after(DevScalars *__restrict__ sc, CgState &s)
{
    for (int j = 0; j < GP_NTR; j++) {
        double J = sc->t_chi2[j] - s.alpha * sc->t_entropy[j];
        if (!isfinite(J)) J = INFINITY;  // a trial that overflows is never the best
        if (s.npts < GP_LS_MAX_PTS) {
            s.pts_s[s.npts] = s.ts[j];
            s.pts_J[s.npts] = J;
            s.npts++;
        }
    }
    s.criterion_evals += GP_NTR;
    s.batches++;
    s.bround++;
    // best point (ties: the smaller step) against the current image (s = 0)
    int b = -1;
    double sb = 0.0, Jb = s.J_init;
    for (int i = 0; i < s.npts; i++) {
        const double Ji = s.pts_J[i], si = s.pts_s[i];
        if (Ji < Jb || (Ji == Jb && b >= 0 && si < sb)) {
            b = i;
            sb = si;
            Jb = Ji;
        }
    }
    if (b < 0) {
        // no trial decreased J: move the grid below the smallest step tried
        double smin = s.pts_s[0];
        for (int i = 1; i < s.npts; i++) smin = fmin(smin, s.pts_s[i]);
        if (s.bround < GP_LS_MAX_ROUNDS && smin > 1e-300) {
            s.s_c = ldexp(smin, -5 * GP_LS_RATIO_LOG2);  // smin / 4^5
            ls_batch_grid(s);
        } else {
            s.force_sd = 1;  // restart from steepest descent next iteration
            ls_batch_accept(s, 0.0, s.J_init);
        }
        return;
    }
    double lo = 0.0, hi = INFINITY;
    for (int i = 0; i < s.npts; i++) {
        const double si = s.pts_s[i];
        if (si < sb && si > lo) lo = si;
        if (si > sb && si < hi) hi = si;
    }
    if (!(hi < INFINITY)) {
        // the largest step tried is the best: extend the grid upwards
        if (s.bround < GP_LS_MAX_ROUNDS - 1 && sb < s.batch_step_max) {
            s.s_c = ldexp(sb, 4 * GP_LS_RATIO_LOG2);  // sb 4^4
            ls_batch_grid(s);
        } else {
            ls_batch_accept(s, sb, Jb);
        }
        return;
    }
    if (s.bphase == BR_GRID && s.bround < GP_LS_MAX_ROUNDS) {
        s.bphase = BR_REFINE;
        for (int j = 0; j < GP_NTR; j++) s.ts[j] = lo + (hi - lo) * (double)(j + 1) / (double)(GP_NTR + 1);
        s.action = CG_EVAL_BATCH;
        return;
    }
    ls_batch_accept(s, sb, Jb);
}

// Projected L-BFGS, candidate pair: accept it when s.y > 1e-12 |s| |y| (the
// newest GP_LB_PAIRS are kept, the oldest is evicted), record its dots in the
// Gram matrices and take gamma from it; a failed batched search drops the
// history afterwards.
__device__ void lb_after_pair(DevScalars *__restrict__ sc, CgState &s)
{
    const double *pd = sc->lb_pdots;
    if (s.lb_xvalid) {
        const double sy = pd[0], yy = pd[1], ss = pd[2];
        if (yy > 0.0 && sy > 1e-12 * sqrt(ss * yy)) {
            const int m = s.lb_count;
            double sy_col[GP_LB_PAIRS], yy_col[GP_LB_PAIRS];  // stored pair i with the new y
            for (int i = 0; i < m; i++) {
                sy_col[i] = pd[3 + i];
                yy_col[i] = pd[3 + GP_LB_PAIRS + i];
            }
            const int cand = s.lb_slot[GP_LB_PAIRS];
            int base = 0, mm = m;
            if (m == GP_LB_PAIRS) {
                // evict the oldest: its buffer becomes the free one
                const int old = s.lb_slot[0];
                for (int i = 0; i + 1 < GP_LB_PAIRS; i++) s.lb_slot[i] = s.lb_slot[i + 1];
                s.lb_slot[GP_LB_PAIRS] = old;
                for (int i = 0; i + 1 < GP_LB_PAIRS; i++)
                    for (int j = 0; j + 1 < GP_LB_PAIRS; j++) {
                        s.lb_sy[i][j] = s.lb_sy[i + 1][j + 1];
                        s.lb_yy[i][j] = s.lb_yy[i + 1][j + 1];
                    }
                base = 1;
                mm = GP_LB_PAIRS - 1;
            } else {
                s.lb_slot[GP_LB_PAIRS] = s.lb_slot[m];
            }
            s.lb_slot[mm] = cand;
            for (int i = 0; i < mm; i++) {
                s.lb_sy[i][mm] = sy_col[i + base];
                s.lb_yy[i][mm] = yy_col[i + base];
                s.lb_yy[mm][i] = yy_col[i + base];
            }
            s.lb_sy[mm][mm] = sy;
            s.lb_yy[mm][mm] = yy;
            s.lb_gamma = sy / yy;
            s.lb_count = mm + 1;
        }
    }
    if (s.lb_drop) {
        s.lb_count = 0;
        s.lb_drop = 0;
    }
}

// Projected L-BFGS, direction coefficients from the compact form; with the
// reference's search, a direction that is not a descent direction is replaced
// by the projected -g at once (the batched search restarts the next iteration
// instead, as for CG).
__device__ void lb_coefficients(DevScalars *__restrict__ sc, CgState &s)
{
    const double *qd = sc->lb_qdots;
    const int m = s.lb_count;
    for (int i = 0; i < GP_LB_PAIRS; i++) {
        s.lb_cs[i] = 0.0;
        s.lb_cy[i] = 0.0;
    }
    s.lb_cq = 1.0;
    if (m == 0) return;
    const double gam = s.lb_gamma;
    double x[GP_LB_PAIRS], z[GP_LB_PAIRS], t[GP_LB_PAIRS];
    // R x = u (R upper triangular, R_ij = s_i.y_j for i <= j)
    for (int i = m - 1; i >= 0; i--) {
        double v = qd[1 + i];
        for (int j = i + 1; j < m; j++) v -= s.lb_sy[i][j] * x[j];
        x[i] = v / s.lb_sy[i][i];
    }
    // z = (D + gamma Y Y^T) x - gamma Y q
    for (int i = 0; i < m; i++) {
        double v = s.lb_sy[i][i] * x[i];
        for (int j = 0; j < m; j++) v += gam * s.lb_yy[i][j] * x[j];
        z[i] = v - gam * qd[1 + GP_LB_PAIRS + i];
    }
    // R^T t = z
    for (int i = 0; i < m; i++) {
        double v = z[i];
        for (int j = 0; j < i; j++) v -= s.lb_sy[j][i] * t[j];
        t[i] = v / s.lb_sy[i][i];
    }
    double w1 = gam * qd[0];
    for (int i = 0; i < m; i++) {
        s.lb_cs[i] = t[i];
        s.lb_cy[i] = -gam * x[i];
        w1 += t[i] * qd[1 + i] - gam * x[i] * qd[1 + GP_LB_PAIRS + i];
    }
    s.lb_cq = gam;
    // d.g = -w1: not a descent direction (or not finite) with the reference's search -> projected -g
    if (s.ls_mode != GPAIR_LS_BATCH && !(w1 > 0.0)) {
        s.lb_count = 0;
        for (int i = 0; i < GP_LB_PAIRS; i++) {
            s.lb_cs[i] = 0.0;
            s.lb_cy[i] = 0.0;
        }
        s.lb_cq = 1.0;
    }
}

// One step of the CG state machine.
__device__ __noinline__ static void cg_step(DevScalars *__restrict__ sc, CgState &s, int what)
{
    switch (what) {
    case CTRL_RESUME:
        // a continued run counts its own evaluations; the iteration state is kept
        s.criterion_evals = s.grad_evals = 0;
        s.batches = 0;
        s.run_it = 0;
        s.reached = 0;
        s.stopped = 0;
        sc->nonfinite = 0;
        break;
    case CTRL_AFTER_BATCH:
        if (sc->tc_err) {
            s.sel = 0.0;
            s.action = CG_DONE;
            break;
        }
        ls_batch_after(sc, s);
        break;
    case CTRL_END:
        s.run_it++;
        break;
    case CTRL_LB_PAIR:
        lb_after_pair(sc, s);
        break;
    case CTRL_LB_COEF:
        lb_coefficients(sc, s);
        break;
    case CTRL_INIT:
        s.run_it = 0;
        s.it = 0;
        s.criterion_evals = s.grad_evals = 0;
        s.batches = 0;
        s.beta = 0.0;
        s.sel = 0.0;
        s.prev_nn = 0.0;
        s.action = CG_EVAL_CRIT;
        s.s_c = 1.0;
        s.reached = 0;
        s.stopped = 0;
        s.force_sd = 0;
        sc->nonfinite = 0;
        s.lb_count = 0;
        s.lb_xvalid = 0;
        s.lb_drop = 0;
        s.lb_gamma = 1.0;
        for (int i = 0; i <= GP_LB_PAIRS; i++) s.lb_slot[i] = i;
        break;
    case CTRL_BEGIN: {
        // criterion and gradient of the current image are done (gpair.c:688-724);
        // beta from the FP64 dot products of the gradient finalize (gpair.c:727-758)
        s.J = sc->chi2 - s.alpha * sc->entropy;
        s.chi2 = sc->chi2;
        s.entropy = sc->entropy;
        s.criterion_evals++;
        s.grad_evals++;
        const double nn = sc->grad_dots[0][0], no = sc->grad_dots[0][1];
        const double dn = sc->grad_dots[0][2], dold = sc->grad_dots[0][3];
        const double oo = s.prev_nn;
        double beta = 0.0;
        if (!(s.it == 0 || s.method == 0)) {
            if (s.method == 1) beta = nn / oo;
            if (s.method == 2) {
                beta = (nn - no) / oo;
                if (beta < 0.0) beta = 0.0;
            }
            if (s.method == 3) {
                beta = (nn - no) / (dn - dold);
                if (beta < 0.0) beta = 0.0;
            }
            if (fabs(no / nn) > 0.5) beta = 0.0;
        }
        if (s.force_sd) {
            beta = 0.0;
            s.force_sd = 0;
            if (s.method == 4) s.lb_drop = 1;  // projected L-BFGS: the history goes after this pair
        }
        s.beta = beta;
        s.prev_nn = nn;
        s.it++;
        if (s.target_J > 0.0 && s.J <= s.target_J) {
            s.reached = 1;
            if (sc->stop_flag) atomicExch(sc->stop_flag, 1);  // tell the runs racing this one
        } else if (sc->stop_flag && *(volatile int *)sc->stop_flag) {
            s.stopped = 1;
        }
        break;
    }
    case CTRL_AFTER_DIR:
        if (s.reached || s.stopped) {  // target reached here or by a racing run: the run ends here
            s.sel = 0.0;
            s.action = CG_DONE;
            break;
        }
        if (s.ls_mode == GPAIR_LS_BATCH) {
            s.wolfe1 = sc->dir_dot;
            s.J_init = s.J;
            s.sel = 0.0;
            s.npts = 0;
            s.bround = 0;
            s.bphase = BR_GRID;
            if (s.method == 4) s.lb_xvalid = 1;  // the combination pass saved x_old
            if (!(s.wolfe1 < 0.0)) {  // not a descent direction: restart from -g
                s.force_sd = 1;
                s.action = CG_DONE;
                break;
            }
            // a quasi-Newton direction carries its own scale: grid centred on step 1
            if (s.method == 4 && s.lb_count > 0) s.s_c = 1.0;
            if (!(s.s_c > 0.0) || !isfinite(s.s_c)) s.s_c = 1.0;
            ls_batch_grid(s);
            break;
        }
        // line search initialisation (gpair.c:792-806)
        if (s.method == 4) s.lb_xvalid = 1;
        s.wolfe1 = sc->dir_dot;
        s.sel = 0.0;
        s.s = 1.0;
        s.s_old = 0.0;
        s.J_init = s.J;
        s.J_old = s.J;
        s.ls_it = 1;
        s.phase = CG_PH_BRACKET;
        s.bracket_trials = 0;
        s.action = CG_EVAL_CRIT;
        break;
    case CTRL_AFTER_CRIT: {
        if (sc->tc_err) {  // a tensor-core kernel gave up a bounded wait: stop the run
            s.sel = 0.0;
            s.action = CG_DONE;
            break;
        }
        double Jt = sc->chi2 - s.alpha * sc->entropy;
        s.Jt = Jt;
        s.criterion_evals++;
        if (s.phase == CG_PH_BRACKET) {
            // gpair.c:832-849
            if ((Jt > (s.J_init + s.c1 * s.s * s.wolfe1)) || ((Jt >= s.J_old) && (s.ls_it > 1)))
                cg_zoom_enter(s, s.s_old, s.s, s.J_old);
            else
                s.action = CG_EVAL_GRAD;
        } else {
            // gpu.c:2019-2023
            if ((Jt > (s.J_init + s.c1 * s.z_s * s.wolfe1)) || (Jt >= s.J_lo)) {
                s.hi = s.z_s;
                s.z_s_old = s.z_s;
                s.z_J_old = Jt;
                s.zoom_counter++;
                cg_zoom_next(s);
            } else {
                s.action = CG_EVAL_GRAD;
            }
        }
        if (!isfinite(Jt)) {
            sc->nonfinite |= 8u;
            s.sel = 0.0;
            s.action = CG_DONE;
        }
        break;
    }
    case CTRL_AFTER_GRAD: {
        if (sc->tc_err) {
            s.sel = 0.0;
            s.action = CG_DONE;
            break;
        }
        const double w2 = sc->grad_dots[1][2];  // d . g_trial
        s.grad_evals++;
        if (s.phase == CG_PH_BRACKET) {
            // gpair.c:861-903
            if (fabs(w2) <= -s.c2 * s.wolfe1) {
                s.sel = s.s;
                s.action = CG_DONE;
            } else if (w2 >= 0.0) {
                cg_zoom_enter(s, s.s, s.s_old, s.Jt);
            } else {
                s.s_old = s.s;
                s.J_old = s.Jt;
                s.s = 10.0 * s.s;
                if (s.s > s.step_max) s.s = s.step_max;
                s.ls_it++;
                s.bracket_trials++;
                s.action = (s.bracket_trials >= s.max_bracket) ? CG_DONE : CG_EVAL_CRIT;
                if (s.action == CG_DONE) s.sel = s.s_old;
            }
        } else {
            // gpu.c:2036-2056
            if ((w2 >= s.c2 * s.wolfe1) || (s.zoom_counter > 10)) {
                s.sel = s.z_s;
                s.action = CG_DONE;
            } else {
                if (w2 * (s.hi - s.lo) >= 0.0) s.hi = s.lo;
                s.lo = s.z_s;
                s.z_s_old = s.z_s;
                s.z_J_old = s.Jt;
                s.zoom_counter++;
                cg_zoom_next(s);
            }
        }
        break;
    }
    default:
        break;
    }
}

// The controller runs in one thread at the end of a reduction kernel, on the
// critical path of every evaluation. The state machine stays out of line so
// that its registers do not count against the reduction kernels' occupancy,
// and it works on the device-global state in place: a copy of the 1 KB state
// to local memory and back made the one-thread controller about four times
// slower (9 us instead of 2 us per launch).
__device__ void cg_control(DevScalars *__restrict__ sc, int what) { cg_step(sc, sc->cg, what); }

__global__ void k_cg_ctrl(DevScalars *__restrict__ sc, int what)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    cg_control(sc, what);
}

// Graph-captured controller: runs the same state machine, then steers the CG
// graph: h_ls keeps the line-search loop going, h_grad selects the gradient
// branch of a trial, h_iter keeps the iteration loop going. At the end of an
// iteration it appends (J, chi2, S, step, beta) to the device trace.
__device__ void cg_set_handles(DevScalars *__restrict__ sc, int what, cudaGraphConditionalHandle h_iter,
                               cudaGraphConditionalHandle h_ls, cudaGraphConditionalHandle h_grad)
{
    const CgState &s = sc->cg;
    switch (what) {
    case CTRL_AFTER_DIR:
    case CTRL_AFTER_BATCH:
        cudaGraphSetConditional(h_ls, s.action != CG_DONE ? 1u : 0u);
        break;
    case CTRL_AFTER_CRIT:
        cudaGraphSetConditional(h_grad, s.action == CG_EVAL_GRAD ? 1u : 0u);
        cudaGraphSetConditional(h_ls, s.action != CG_DONE ? 1u : 0u);
        break;
    case CTRL_AFTER_GRAD:
        cudaGraphSetConditional(h_ls, s.action != CG_DONE ? 1u : 0u);
        break;
    case CTRL_END:
        cudaGraphSetConditional(h_iter, cg_run_goes_on(sc) ? 1u : 0u);
        break;
    default:
        break;
    }
}

// Graph-captured controller: runs the same state machine, then steers the CG
// graph: h_ls keeps the line-search loop going, h_grad selects the gradient
// branch of a trial, h_iter keeps the iteration loop going. At the end of an
// iteration it appends (J, chi2, S, step, beta) to the device trace.
struct CtrlArgs {
    DevScalars *sc;
    int what;
    cudaGraphConditionalHandle h_iter, h_ls, h_grad;
    double *trace;
    int trace_cap;
    GP_VGRID_FIELDS;
};

__device__ __forceinline__ void cg_ctrl_g_body(const CtrlArgs &A, const GpVGrid &vg)
{
    if (threadIdx.x != 0 || vg.bx != 0) return;
    DevScalars *__restrict__ sc = A.sc;
    CgState &s = sc->cg;
    if (A.what == CTRL_END && s.run_it < A.trace_cap && A.trace) {
        double *t = A.trace + 5 * (size_t)s.run_it;
        t[0] = s.J;
        t[1] = s.chi2;
        t[2] = s.entropy;
        t[3] = s.sel;
        t[4] = s.beta;
    }
    cg_control(sc, A.what);
    if (A.h_iter) cg_set_handles(sc, A.what, A.h_iter, A.h_ls, A.h_grad);
}

__global__ void k_cg_ctrl_g(const CtrlArgs a)
{
    gp_pdl_enter();
    cg_ctrl_g_body(a, gp_vgrid_hw());
}

struct CtrlOp {
    using Args = CtrlArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { cg_ctrl_g_body(a, v); }
};

int gp_cg_kernel_graph(gpair_ctx *c, int which_ctrl, unsigned long long h_iter, unsigned long long h_ls,
                       unsigned long long h_grad, double *trace, int trace_cap)
{
    const CtrlArgs a = {c->sc, which_ctrl, h_iter, h_ls, h_grad, trace, trace_cap, 1, 1};
    GP_LAUNCH(c, gp_launch(c, k_cg_ctrl_g, dim3(1), dim3(32), 0, a));
    return GPAIR_OK;
}

int gp_cg_kernel(gpair_ctx *c, int which_ctrl)
{
    k_cg_ctrl<<<1, 32, 0, c->stream>>>(c->sc, which_ctrl);
    GP_LAUNCH_CHECK(c);
    return GPAIR_OK;
}

// ------------------------------------------------- grouped stage launches
//
// Lockstep batches run each stage of an iteration as one launch over all their
// instances (group.cuh): the argument structs below are built by the same
// functions as the single launches, with the controller step each stage takes
// in a lockstep iteration and no graph handles (the batch's routers steer).

static FusedCtrl ctrl_only(int what)
{
    FusedCtrl f;
    memset(&f, 0, sizeof(f));
    f.what = what;
    return f;
}

size_t gp_stage_args_size(int stage)
{
    switch (stage) {
    case GS_VIS_DATA: return sizeof(VisDataArgs);
    case GS_ADJ_WEIGHTS: return sizeof(AdjWeightsArgs);
    case GS_GRAD_FINALIZE: return sizeof(GradFinalizeArgs);
    case GS_DESCENT: return sizeof(DescentArgs);
    case GS_CHI2_BATCH: return sizeof(VisChi2BatchArgs);
    case GS_UPDATE: return sizeof(UpdateImageArgs);
    case GS_CTRL_END: return sizeof(CtrlArgs);
    default: return gp_tc_stage_args_size(stage);
    }
}

template <class A>
static int put_args(const A &a, void *out, int *nblocks)
{
    memcpy(out, &a, sizeof(A));
    *nblocks = a.nbx * a.nby;
    return GPAIR_OK;
}

int gp_stage_args(gpair_ctx *c, int stage, double *trace, void *out, int *nblocks)
{
    switch (stage) {
    case GS_VIS_DATA: return put_args(vis_data_args(c, 0, ctrl_only(-1)), out, nblocks);
    case GS_ADJ_WEIGHTS: return put_args(adj_weights_args(c), out, nblocks);
    case GS_GRAD_FINALIZE:
        return put_args(grad_finalize_args(c, GPAIR_IMG_CURR, GRAD_FUSED, -1.f, ctrl_only(CTRL_BEGIN)), out, nblocks);
    case GS_DESCENT: return put_args(descent_args(c, 1, 0.0, ctrl_only(CTRL_AFTER_DIR)), out, nblocks);
    case GS_CHI2_BATCH:
        return put_args(batch_chi2_args(c, c->epp, ctrl_only(CTRL_AFTER_BATCH), nullptr), out, nblocks);
    case GS_UPDATE: return put_args(update_image_args(c, 1, 0.0, 1e-8, 1), out, nblocks);
    case GS_CTRL_END: {
        const CtrlArgs a = {c->sc, CTRL_END, 0, 0, 0, trace, 1, 1, 1};
        return put_args(a, out, nblocks);
    }
    default: return GPAIR_ERR_INVALID;
    }
}

template <class Op, int THREADS>
static int group_launch(gpair_ctx *c, const void *d_args, const int *d_start, int n, int total, const int *gate)
{
    GP_LAUNCH(c, gp_launch(c, k_grouped<Op, THREADS>, dim3(total), dim3(THREADS), 0,
                           (const typename Op::Args *)d_args, d_start, n, gate));
    return GPAIR_OK;
}

int gp_stage_group_launch(gpair_ctx *c, int stage, const void *d_args, const int *d_start, int n, int total,
                          const int *gate)
{
    if (total < 1 || n < 1) return GPAIR_ERR_INVALID;
    switch (stage) {
    case GS_VIS_DATA: return group_launch<VisDataOp, GP_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_ADJ_WEIGHTS: return group_launch<AdjWeightsOp, GP_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_GRAD_FINALIZE: return group_launch<GradFinalizeOp, GP_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_DESCENT: return group_launch<DescentOp, GP_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_CHI2_BATCH: return group_launch<VisChi2BatchOp, GP_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_UPDATE: return group_launch<UpdateImageOp, 256>(c, d_args, d_start, n, total, gate);
    case GS_CTRL_END: return group_launch<CtrlOp, 32>(c, d_args, d_start, n, total, gate);
    default: return GPAIR_ERR_INVALID;
    }
}
