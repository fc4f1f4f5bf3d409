// warmstart_cnn.cu -- training and inference kernels of the warm-start
// network: a 4-level convolutional encoder/decoder that maps per-problem
// feature maps (dirty images and the gridded uv density) to a positive,
// unit-flux start image for CG.
//
// The reference has no learned component; these kernels serve the
// library's warm-start extension only. Layout: activations float NCHW
// [B][C][H][W]; 3x3 weights [Cout][Cin][3][3] as bf16 (the layer's working
// copy of an FP32 master), FP32 accumulation everywhere, FP64 for the
// per-image normalisation and loss sums. All reductions are deterministic
// (per-block partials summed in a fixed order, no floating-point atomics).
//
//   k_conv3       3x3 convolution, zero padding: bias, optional residual add,
//                 optional ReLU. With `flip` it is the data-gradient of a
//                 convolution (transposed, flipped taps; input channels =
//                 the forward's output channels), optionally accumulating.
//   k_conv3_wgrad per-slice partials of dW[co][ci][tap] and db[co]
//   k_reduce_slices  fixed-order sum of those partials
//   k_relu_mask   g *= (y > 0)
//   k_pool2 / k_pool2_bwd / k_up2 / k_up2_bwd   2x2 average pool, nearest upsample
//   k_head / k_head_bwd  1x1 conv -> softplus -> divide by the image sum
//   k_mse         per-image squared error (absolute or relative), gradient
//   k_adam        Adam step on FP32 masters, bf16 working copy
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "gpair_b200.h"

#define CV_T 16    // output tile edge (pixels)
#define CV_CO 16   // output channels per block
#define CV_CI 8    // input channels per shared-memory chunk
#define WG_CI 8    // input channels per weight-gradient block
#define NTAP 9

__device__ __forceinline__ float bf(const __nv_bfloat16 *w, size_t i) { return __bfloat162float(w[i]); }

// out[b][co][y][x] = act(bias[co] + skip + sum_ci,tap w * in[b][ci][y+dy][x+dx])
// flip: in = dL/d(out) of a forward conv with weights w[Cin][Cout][3][3]
// (here Cin/Cout are the forward's Cout/Cin), taps mirrored.
__global__ void __launch_bounds__(CV_T *CV_T) k_conv3(const float *__restrict__ in, const __nv_bfloat16 *__restrict__ w,
                                                       const float *__restrict__ bias, const float *__restrict__ skip,
                                                       float *__restrict__ out, int Cin, int Cout, int H, int W,
                                                       int relu, int flip, int accumulate)
{
    __shared__ float xs[CV_CI][CV_T + 2][CV_T + 2];
    __shared__ float ws[CV_CO][CV_CI][NTAP];
    const int tiles_x = (W + CV_T - 1) / CV_T;
    const int tx0 = (blockIdx.x % tiles_x) * CV_T, ty0 = (blockIdx.x / tiles_x) * CV_T;
    const int co0 = blockIdx.y * CV_CO, b = blockIdx.z;
    const int tx = threadIdx.x % CV_T, ty = threadIdx.x / CV_T;
    const int x = tx0 + tx, y = ty0 + ty;
    const float *inb = in + (size_t)b * Cin * H * W;
    float acc[CV_CO];
#pragma unroll
    for (int i = 0; i < CV_CO; i++) acc[i] = 0.f;
    for (int ci0 = 0; ci0 < Cin; ci0 += CV_CI) {
        // input tile with a one-pixel halo, zero outside the image
        for (int i = threadIdx.x; i < CV_CI * (CV_T + 2) * (CV_T + 2); i += blockDim.x) {
            const int c = i / ((CV_T + 2) * (CV_T + 2)), r = i % ((CV_T + 2) * (CV_T + 2));
            const int yy = ty0 - 1 + r / (CV_T + 2), xx = tx0 - 1 + r % (CV_T + 2);
            float v = 0.f;
            if (ci0 + c < Cin && yy >= 0 && yy < H && xx >= 0 && xx < W) v = inb[((size_t)(ci0 + c) * H + yy) * W + xx];
            xs[c][r / (CV_T + 2)][r % (CV_T + 2)] = v;
        }
        for (int i = threadIdx.x; i < CV_CO * CV_CI * NTAP; i += blockDim.x) {
            const int o = i / (CV_CI * NTAP), c = (i / NTAP) % CV_CI, k = i % NTAP;
            float v = 0.f;
            if (co0 + o < Cout && ci0 + c < Cin) {
                if (!flip) v = bf(w, ((size_t)(co0 + o) * Cin + ci0 + c) * NTAP + k);
                else v = bf(w, ((size_t)(ci0 + c) * Cout + co0 + o) * NTAP + (NTAP - 1 - k));
            }
            ws[o][c][k] = v;
        }
        __syncthreads();
#pragma unroll 2
        for (int c = 0; c < CV_CI; c++) {
            float v[NTAP];
#pragma unroll
            for (int k = 0; k < NTAP; k++) v[k] = xs[c][ty + k / 3][tx + k % 3];
#pragma unroll
            for (int o = 0; o < CV_CO; o++) {
                float a = acc[o];
#pragma unroll
                for (int k = 0; k < NTAP; k++) a = fmaf(ws[o][c][k], v[k], a);
                acc[o] = a;
            }
        }
        __syncthreads();
    }
    if (x >= W || y >= H) return;
#pragma unroll
    for (int o = 0; o < CV_CO; o++) {
        const int co = co0 + o;
        if (co >= Cout) break;
        const size_t idx = (((size_t)b * Cout + co) * H + y) * W + x;
        float v = acc[o] + (bias ? bias[co] : 0.f);
        if (skip) v += skip[idx];
        if (relu) v = fmaxf(v, 0.f);
        out[idx] = accumulate ? out[idx] + v : v;
    }
}

// Weight and bias gradient partials: block (co, ci-chunk, slice) sums over the
// images [slice*bps, (slice+1)*bps) and all pixels; part[slice][co][ci][tap],
// bpart[slice][co] (bias, from the ci-chunk 0 blocks).
__global__ void __launch_bounds__(256) k_conv3_wgrad(const float *__restrict__ in, const float *__restrict__ g,
                                                     float *__restrict__ part, float *__restrict__ bpart, int B,
                                                     int Cin, int Cout, int H, int W, int bps)
{
    __shared__ float red[8][WG_CI * NTAP + 1];
    const int co = blockIdx.x, ci0 = blockIdx.y * WG_CI, slice = blockIdx.z;
    const int b0 = slice * bps, b1 = min(B, b0 + bps);
    float acc[WG_CI * NTAP + 1];
#pragma unroll
    for (int i = 0; i < WG_CI * NTAP + 1; i++) acc[i] = 0.f;
    const int HW = H * W;
    for (int b = b0; b < b1; b++) {
        const float *gb = g + ((size_t)b * Cout + co) * HW;
        const float *ib = in + (size_t)b * Cin * HW;
        for (int p = threadIdx.x; p < HW; p += blockDim.x) {
            const float gv = gb[p];
            acc[WG_CI * NTAP] += gv;
            if (gv == 0.f) continue;
            const int y = p / W, x = p - y * W;
#pragma unroll
            for (int k = 0; k < NTAP; k++) {
                const int yy = y + k / 3 - 1, xx = x + k % 3 - 1;
                if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
#pragma unroll
                for (int c = 0; c < WG_CI; c++)
                    if (ci0 + c < Cin) acc[c * NTAP + k] = fmaf(gv, ib[(size_t)(ci0 + c) * HW + yy * W + xx], acc[c * NTAP + k]);
            }
        }
    }
    // fixed-order block reduction: warp shuffles, then one pass over the 8 warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < WG_CI * NTAP + 1; i++) {
        float v = acc[i];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][i] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < WG_CI * NTAP + 1; i += blockDim.x) {
        float v = 0.f;
        for (int w8 = 0; w8 < (int)(blockDim.x >> 5); w8++) v += red[w8][i];
        if (i < WG_CI * NTAP) {
            const int c = i / NTAP, k = i % NTAP;
            if (ci0 + c < Cin) part[(((size_t)slice * Cout + co) * Cin + ci0 + c) * NTAP + k] = v;
        } else if (blockIdx.y == 0) {
            bpart[(size_t)slice * Cout + co] = v;
        }
    }
}

// out[i] = sum over slices of part[s][i] (fixed order)
__global__ void k_reduce_slices(const float *__restrict__ part, int n, int slices, float *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int k = 0; k < slices; k++) s += part[(size_t)k * n + i];
    out[i] = s;
}

__global__ void k_relu_mask(const float *__restrict__ y, float *__restrict__ g, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(y[i] > 0.f)) g[i] = 0.f;
}

// 2x2 average pool: in [BC][H][W] -> out [BC][H/2][W/2]
__global__ void k_pool2(const float *__restrict__ in, float *__restrict__ out, long long BC, int H, int W)
{
    const int Ho = H / 2, Wo = W / 2;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BC * Ho * Wo) return;
    const long long bc = i / (Ho * Wo);
    const int r = (int)(i % (Ho * Wo)), y = r / Wo, x = r % Wo;
    const float *p = in + (size_t)bc * H * W + (size_t)(2 * y) * W + 2 * x;
    out[i] = 0.25f * ((p[0] + p[1]) + (p[W] + p[W + 1]));
}

__global__ void k_pool2_bwd(const float *__restrict__ gout, float *__restrict__ gin, long long BC, int H, int W,
                            int accumulate)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BC * H * W) return;
    const long long bc = i / (H * W);
    const int r = (int)(i % (H * W)), y = r / W, x = r % W;
    const float v = 0.25f * gout[(size_t)bc * (H / 2) * (W / 2) + (y / 2) * (W / 2) + x / 2];
    gin[i] = accumulate ? gin[i] + v : v;
}

// nearest 2x upsample: in [BC][H][W] -> out [BC][2H][2W]
__global__ void k_up2(const float *__restrict__ in, float *__restrict__ out, long long BC, int H, int W)
{
    const int Ho = 2 * H, Wo = 2 * W;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BC * Ho * Wo) return;
    const long long bc = i / (Ho * Wo);
    const int r = (int)(i % (Ho * Wo)), y = r / Wo, x = r % Wo;
    out[i] = in[(size_t)bc * H * W + (y / 2) * W + x / 2];
}

__global__ void k_up2_bwd(const float *__restrict__ gout, float *__restrict__ gin, long long BC, int H, int W)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= BC * H * W) return;
    const long long bc = i / (H * W);
    const int r = (int)(i % (H * W)), y = r / W, x = r % W;
    const float *p = gout + (size_t)bc * 4 * H * W + (size_t)(2 * y) * (2 * W) + 2 * x;
    gin[i] = (p[0] + p[1]) + (p[2 * W] + p[2 * W + 1]);
}

__device__ __forceinline__ float softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

__device__ double block_sum_d(double v, double *sm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    __syncthreads();
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < nw; i++) t += sm[i];
    __syncthreads();
    if (threadIdx.x == 0) sm[0] = t;
    __syncthreads();
    t = sm[0];
    __syncthreads();
    return t;
}

// Head, one block per image: z = w . d + bias, a = softplus(z), out = a / sum(a)
__global__ void __launch_bounds__(256) k_head(const float *__restrict__ d, const float *__restrict__ w,
                                              const float *__restrict__ bias_p, float *__restrict__ z,
                                              float *__restrict__ out, float *__restrict__ asum, int C, int HW)
{
    __shared__ double sm[32];
    const int b = blockIdx.x;
    const float bias = *bias_p;
    const float *db = d + (size_t)b * C * HW;
    double s = 0.0;
    for (int p = threadIdx.x; p < HW; p += blockDim.x) {
        float v = bias;
        for (int c = 0; c < C; c++) v = fmaf(w[c], db[(size_t)c * HW + p], v);
        z[(size_t)b * HW + p] = v;
        s += (double)softplus(v);
    }
    s = block_sum_d(s, sm);
    const float inv = (float)(1.0 / s);
    for (int p = threadIdx.x; p < HW; p += blockDim.x) out[(size_t)b * HW + p] = softplus(z[(size_t)b * HW + p]) * inv;
    if (threadIdx.x == 0) asum[b] = (float)s;
}

// Head backward, one block per image: gz = ((gout - <gout, out>) / S) sigmoid(z),
// gd[b][c][p] = w[c] gz, and per-image partials of dw[c] (c < C) and dbias (c = C).
__global__ void __launch_bounds__(256) k_head_bwd(const float *__restrict__ d, const float *__restrict__ w,
                                                  const float *__restrict__ z, const float *__restrict__ out,
                                                  const float *__restrict__ asum, const float *__restrict__ gout,
                                                  float *__restrict__ gd, float *__restrict__ part, int C, int HW)
{
    __shared__ double sm[32];
    const int b = blockIdx.x;
    const size_t o = (size_t)b * HW;
    double dot = 0.0;
    for (int p = threadIdx.x; p < HW; p += blockDim.x) dot += (double)gout[o + p] * out[o + p];
    dot = block_sum_d(dot, sm);
    const float invS = 1.f / asum[b], fd = (float)dot;
    const float *db = d + (size_t)b * C * HW;
    float *gdb = gd + (size_t)b * C * HW;
    for (int c = 0; c <= C; c++) {
        double s = 0.0;
        for (int p = threadIdx.x; p < HW; p += blockDim.x) {
            const float gz = (gout[o + p] - fd) * invS * sigmoid(z[o + p]);
            if (c < C) {
                s += (double)gz * db[(size_t)c * HW + p];
                gdb[(size_t)c * HW + p] = w[c] * gz;
            } else {
                s += gz;
            }
        }
        s = block_sum_d(s, sm);
        if (threadIdx.x == 0) part[(size_t)b * (C + 1) + c] = (float)s;
    }
}

// Per-image loss and its gradient (x gscale), FP64 sums:
//   mode 0: npix * sum_p (out - t)^2                 g = 2 npix (out - t)
//   mode 1: sum_p (out - t)^2 / sum_p t^2 (relative)  g = 2 (out - t) / sum_p t^2
__global__ void __launch_bounds__(256) k_mse(const float *__restrict__ out, const float *__restrict__ t,
                                             float *__restrict__ g, double *__restrict__ loss, int HW, float gscale,
                                             int mode)
{
    __shared__ double sm[32];
    const int b = blockIdx.x;
    const size_t o = (size_t)b * HW;
    double tt = 1.0;
    if (mode == 1) {
        double s2 = 0.0;
        for (int p = threadIdx.x; p < HW; p += blockDim.x) s2 += (double)t[o + p] * t[o + p];
        tt = block_sum_d(s2, sm);
        if (!(tt > 0.0)) tt = 1.0;
    }
    const float f = mode == 1 ? (float)(2.0 / tt) : 2.f * (float)HW;
    double s = 0.0;
    for (int p = threadIdx.x; p < HW; p += blockDim.x) {
        const float e = out[o + p] - t[o + p];
        s += (double)e * e;
        if (g) g[o + p] = gscale * f * e;
    }
    s = block_sum_d(s, sm);
    if (threadIdx.x == 0) loss[b] = mode == 1 ? s / tt : s * HW;
}

__global__ void k_adam(float *__restrict__ p, __nv_bfloat16 *__restrict__ pbf, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (pbf) pbf[i] = __float2bfloat16_rn(pi);
}

__global__ void k_to_bf16(const float *__restrict__ src, __nv_bfloat16 *__restrict__ dst, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

// ------------------------------------------------------------ C ABI

static inline int cdiv_ll(long long a, long long b) { return (int)((a + b - 1) / b); }
static inline int cnn_status(void) { return cudaGetLastError() == cudaSuccess ? GPAIR_OK : GPAIR_ERR_CUDA; }
#define CNN_STREAM(s) ((cudaStream_t)(s))

extern "C" int gpair_cnn_conv3x3(const float *in, const void *w_bf16, const float *bias, const float *skip, float *out,
                                 int B, int Cin, int Cout, int H, int W, int relu, void *stream)
{
    if (B <= 0 || B > 65535 || Cin <= 0 || Cout <= 0 || H <= 0 || W <= 0) return GPAIR_ERR_INVALID;
    dim3 g(cdiv_ll(W, CV_T) * cdiv_ll(H, CV_T), cdiv_ll(Cout, CV_CO), B);
    k_conv3<<<g, CV_T * CV_T, 0, CNN_STREAM(stream)>>>(in, (const __nv_bfloat16 *)w_bf16, bias, skip, out, Cin, Cout,
                                                       H, W, relu, 0, 0);
    return cnn_status();
}

extern "C" int gpair_cnn_conv3x3_bwd_data(const float *gout, const void *w_bf16, float *gin, int B, int Cin, int Cout,
                                          int H, int W, int accumulate, void *stream)
{
    if (B <= 0 || B > 65535 || Cin <= 0 || Cout <= 0 || H <= 0 || W <= 0) return GPAIR_ERR_INVALID;
    dim3 g(cdiv_ll(W, CV_T) * cdiv_ll(H, CV_T), cdiv_ll(Cin, CV_CO), B);
    k_conv3<<<g, CV_T * CV_T, 0, CNN_STREAM(stream)>>>(gout, (const __nv_bfloat16 *)w_bf16, nullptr, nullptr, gin,
                                                       Cout, Cin, H, W, 0, 1, accumulate);
    return cnn_status();
}

extern "C" int gpair_cnn_conv3x3_bwd_weight(const float *in, const float *gpre, float *dw, float *db, float *scratch,
                                            long long scratch_floats, int B, int Cin, int Cout, int H, int W,
                                            void *stream)
{
    if (B <= 0 || Cin <= 0 || Cout <= 0 || H <= 0 || W <= 0) return GPAIR_ERR_INVALID;
    // about 64K pixels per slice
    int bps = (int)(65536 / ((long long)H * W));
    if (bps < 1) bps = 1;
    if (bps > B) bps = B;
    const int slices = cdiv_ll(B, bps);
    const long long nw = (long long)Cout * Cin * NTAP;
    if ((long long)slices * (nw + Cout) > scratch_floats) return GPAIR_ERR_INVALID;
    float *part = scratch, *bpart = scratch + (size_t)slices * nw;
    dim3 g(Cout, cdiv_ll(Cin, WG_CI), slices);
    k_conv3_wgrad<<<g, 256, 0, CNN_STREAM(stream)>>>(in, gpre, part, bpart, B, Cin, Cout, H, W, bps);
    k_reduce_slices<<<cdiv_ll(nw, 256), 256, 0, CNN_STREAM(stream)>>>(part, (int)nw, slices, dw);
    k_reduce_slices<<<cdiv_ll(Cout, 256), 256, 0, CNN_STREAM(stream)>>>(bpart, Cout, slices, db);
    return cnn_status();
}

extern "C" int gpair_cnn_relu_mask(const float *y, float *g, long long n, void *stream)
{
    if (n <= 0) return GPAIR_ERR_INVALID;
    k_relu_mask<<<cdiv_ll(n, 256), 256, 0, CNN_STREAM(stream)>>>(y, g, n);
    return cnn_status();
}

extern "C" int gpair_cnn_pool2(const float *in, float *out, long long BC, int H, int W, void *stream)
{
    if (BC <= 0 || H < 2 || W < 2 || (H & 1) || (W & 1)) return GPAIR_ERR_INVALID;
    k_pool2<<<cdiv_ll(BC * (H / 2) * (W / 2), 256), 256, 0, CNN_STREAM(stream)>>>(in, out, BC, H, W);
    return cnn_status();
}

extern "C" int gpair_cnn_pool2_bwd(const float *gout, float *gin, long long BC, int H, int W, int accumulate,
                                   void *stream)
{
    if (BC <= 0 || H < 2 || W < 2 || (H & 1) || (W & 1)) return GPAIR_ERR_INVALID;
    k_pool2_bwd<<<cdiv_ll(BC * H * W, 256), 256, 0, CNN_STREAM(stream)>>>(gout, gin, BC, H, W, accumulate);
    return cnn_status();
}

extern "C" int gpair_cnn_up2(const float *in, float *out, long long BC, int H, int W, void *stream)
{
    if (BC <= 0 || H <= 0 || W <= 0) return GPAIR_ERR_INVALID;
    k_up2<<<cdiv_ll(BC * 4 * H * W, 256), 256, 0, CNN_STREAM(stream)>>>(in, out, BC, H, W);
    return cnn_status();
}

extern "C" int gpair_cnn_up2_bwd(const float *gout, float *gin, long long BC, int H, int W, void *stream)
{
    if (BC <= 0 || H <= 0 || W <= 0) return GPAIR_ERR_INVALID;
    k_up2_bwd<<<cdiv_ll(BC * H * W, 256), 256, 0, CNN_STREAM(stream)>>>(gout, gin, BC, H, W);
    return cnn_status();
}

extern "C" int gpair_cnn_head(const float *d, const float *w, const float *bias, float *z, float *out, float *asum,
                              int B, int C, int HW, void *stream)
{
    if (B <= 0 || C <= 0 || HW <= 0) return GPAIR_ERR_INVALID;
    k_head<<<B, 256, 0, CNN_STREAM(stream)>>>(d, w, bias, z, out, asum, C, HW);
    return cnn_status();
}

extern "C" int gpair_cnn_head_bwd(const float *d, const float *w, const float *z, const float *out, const float *asum,
                                  const float *gout, float *gd, float *dw, float *scratch, int B, int C, int HW,
                                  void *stream)
{
    if (B <= 0 || C <= 0 || HW <= 0) return GPAIR_ERR_INVALID;
    k_head_bwd<<<B, 256, 0, CNN_STREAM(stream)>>>(d, w, z, out, asum, gout, gd, scratch, C, HW);
    // dw[c] (c < C) and dbias (c = C): fixed-order sums over the images
    k_reduce_slices<<<1, 256, 0, CNN_STREAM(stream)>>>(scratch, C + 1, B, dw);
    return cnn_status();
}

extern "C" int gpair_cnn_mse(const float *out, const float *target, float *gout, double *loss, int B, int HW,
                             float gscale, int mode, void *stream)
{
    if (B <= 0 || HW <= 0 || mode < 0 || mode > 1) return GPAIR_ERR_INVALID;
    k_mse<<<B, 256, 0, CNN_STREAM(stream)>>>(out, target, gout, loss, HW, gscale, mode);
    return cnn_status();
}

extern "C" int gpair_cnn_adam(float *p, void *p_bf16, const float *g, float *m, float *v, int n, float lr, float b1,
                              float b2, float eps, int step, void *stream)
{
    if (n <= 0 || step <= 0) return GPAIR_ERR_INVALID;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<cdiv_ll(n, 256), 256, 0, CNN_STREAM(stream)>>>(p, (__nv_bfloat16 *)p_bf16, g, m, v, n, lr, b1, b2, eps,
                                                            c1, c2);
    return cnn_status();
}

extern "C" int gpair_cnn_to_bf16(const float *src, void *dst, int n, void *stream)
{
    if (n <= 0) return GPAIR_ERR_INVALID;
    k_to_bf16<<<cdiv_ll(n, 256), 256, 0, CNN_STREAM(stream)>>>(src, (__nv_bfloat16 *)dst, n);
    return cnn_status();
}
